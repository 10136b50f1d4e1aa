// Persistent DFS matcher (replaces gpu_match.cu:96-1119, join.cu:18-221 and
// the work queue of queue.cuh / job_queue.cuh).
//
// One warp per task.  A task fixes positions 0..depth-1 of a matching order
// and enumerates the rest depth-first.  The stack is spread over the lanes:
// lane p keeps the image f[p] of position p with its adjacency run, and the
// iteration state of level p (pivot run, next chunk, pending candidates of the
// current chunk).  Candidates of level p are produced 32 at a time from the
// run of the backward neighbour with the fewest neighbours (the pivot): each
// lane tests one element (label, injectivity, filter bit, membership in the
// other backward neighbours' runs, liveness at the update's view time) and a
// ballot gives the chunk's candidate mask.  Membership in a short range is
// a warp merge over 32-entry tiles, in a long one a binary search; the last
// level of a chunk's candidates is evaluated in one packed pass, with the
// longest shared range staged in shared memory.  Nothing is materialised,
// except, with breadth-first levels, the rows a first launch hands to a
// second.
//
// Scheduling.  Tasks are first the seeds (one atomicAdd each), then donated
// jobs.  An idle warp takes a ticket (one atomicAdd on pop_cnt) and waits for
// its own job slot to be published, polling only that slot's flag with
// exponential backoff.  Busy warps see pop_cnt - push_cnt warps waiting and
// donate to them: pending candidates of their shallowest level with at least
// two levels below it, or half of a long remaining run.  The warp whose task
// completion brings `outstanding` to zero sets `done` and marks every
// still-waiting ticket's slot as finished.  Every wait is bounded by a clock
// budget that restarts whenever busy warps show progress.
#include <algorithm>

#include "kernels.cuh"

namespace dsm {

namespace {

template <class T>
__device__ __forceinline__ T ld_volatile(const T &x) {
  return *(const volatile T *)&x;
}

constexpr unsigned long long kSeqDone = 1ull << 63;

// One candidate of a packed last level: where its pivot range starts in the
// concatenation (excl), its id, its own range of the last level's label
// (run offset in 16-byte units, [a, b)), flags (bit 0: its own range is the
// pivot; bit 1: it is an endpoint of an update of the batch).
struct alignas(16) PackEnt {
  uint32_t excl, cw, off, a, b, flags, pad0, pad1;
};

// Staged probe range of a packed last level (per warp, shared memory): the
// longest last-level range in the run of a fixed position, whole when it has
// at most kStage entries, else every 2^shift-th entry (fences); staged once
// per level-(nq - 2) context, when first packed, if it has kStageMin entries
// or more.  info = lane | shift << 5 | fences << 10, kStageNone: none,
// kStageUnset: not decided yet for this context.
constexpr uint32_t kStage = 512;
constexpr uint32_t kStageMin = 32;
constexpr uint32_t kStageNone = 0xFFFFFFFEu;
constexpr uint32_t kStageUnset = 0xFFFFFFFFu;
struct PackStage {
  uint32_t fence[kStage];
  uint32_t info;
};

// Lane 0 only.  Returns 1 (seed `slot`), 2 (job of ticket `slot`; the caller
// releases the ring slot after reading it) or 0 (no more work).
__device__ uint32_t acquire(const MatchArgs &P, unsigned long long &slot, bool &seeds_done) {
  Sched *sc = P.sc;
  if (!seeds_done) {
    const unsigned long long nseeds = ld_volatile(sc->nseeds);
    if (ld_volatile(sc->seed_next.v) < nseeds) {
      unsigned long long s = atomicAdd(&sc->seed_next.v, 1ull);
      if (s < nseeds) {
        slot = s;
        return 1;
      }
    }
    seeds_done = true;
  }
  const unsigned long long t = atomicAdd(&sc->pop_cnt.v, 1ull);
  __threadfence();
  if (ld_volatile(sc->done.v)) return 0;
  long long t0 = clock64();
  unsigned long long last_prog = ld_volatile(sc->progress.v);
  unsigned ns = 32;
  const unsigned long long *seq = P.job_seq + (t & (P.job_ring - 1));
  for (uint32_t it = 0;; ++it) {
    unsigned long long r = ld_volatile(*seq);
    if (r == t + 1) {
      __threadfence();
      slot = t;
      atomicAdd(&sc->steals, 1ull);
      return 2;
    }
    if (r == (t | kSeqDone)) return 0;
    if ((it & 7) == 7) {
      if (ld_volatile(sc->done.v) || ld_volatile(sc->error)) return 0;
      unsigned long long pr = ld_volatile(sc->progress.v);
      if (pr != last_prog) {
        last_prog = pr;
        t0 = clock64();
      } else if (clock64() - t0 > P.timeout_cycles) {
        atomicOr(&sc->error, kErrTimeout);
        return 0;
      }
    }
    __nanosleep(ns);
    ns = min(ns * 2, 2048u);
  }
}

// Called by the whole warp once its task is finished.
__device__ void finish_task(const MatchArgs &P) {
  const uint32_t lane = threadIdx.x & 31;
  unsigned long long before = 0;
  if (lane == 0) before = atomicAdd(&P.sc->outstanding.v, ~0ull);
  before = __shfl_sync(kFull, before, 0);
  if (before != 1) return;
  // Last task of the launch: release every warp still waiting on a ticket.
  // Every position below push_cnt has been consumed (nothing is outstanding),
  // so the slot of each waiting ticket t is free and holds t; at most one
  // ticket per warp waits, far fewer than the ring's slots.
  unsigned long long lo = 0, hi = 0;
  if (lane == 0) {
    atomicExch(&P.sc->done.v, 1ull);
    __threadfence();
    hi = ld_volatile(P.sc->pop_cnt.v);
    lo = ld_volatile(P.sc->push_cnt.v);
  }
  lo = __shfl_sync(kFull, lo, 0);
  hi = __shfl_sync(kFull, hi, 0);
  for (unsigned long long t = lo + lane; t < hi; t += 32)
    atomicExch(&P.job_seq[t & (P.job_ring - 1)], t | kSeqDone);
}

// kLM: label-major runs with slot offsets (the engine's graph); otherwise
// plain id-sorted runs.  srng[L][j]: for level L and backward neighbour j,
// the range of j's run holding the label of level L (label-major only).
//
// The level being scanned (the current level) keeps its iteration state in
// warp-uniform registers (cur_*), so a chunk reads no lane's state; a level
// with deeper levels running parks its state in lane L (lv_*) and takes it
// back by shuffle when the search returns to it.
//
// Packed last level (label-major runs, P.pack_max > 0).  When a chunk of
// level nq - 2 leaves candidates, the last level of all of them is evaluated
// in one pass.  Candidate k's pivot range is the shortest of the last level's
// backward ranges: those in the runs of fixed positions are the same for every
// candidate (set up with level nq - 2), the one in the candidate's own run is
// its own.  The pivot ranges are laid end to end (an inclusive warp scan of
// their lengths) and scanned 32 entries at a time, each lane finding its
// candidate by a five-step search over the scan, so short sibling ranges fill
// whole chunks instead of one mostly idle chunk each.  When the ranges total
// more than pack_max entries the candidates are expanded one at a time instead,
// where long ranges can be split and donated.
template <bool kLM>
__device__ void run_task(const MatchArgs &P, const DevBatchEdges &bt, uint32_t nupd, uint32_t upd, uint32_t qo,
                         uint32_t depth, uint32_t lo, uint32_t hi, uint32_t fval, uint2 (*srng)[16],
                         PackEnt *spk, PackStage *stg) {
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
  const uint32_t seg = Q.local * nupd + upd;

  uint32_t my_f = fval, my_off = 0, my_deg = 0, my_touch = 0;
  if (lane < depth) {
    uint2 a = P.g.adj[my_f];
    my_off = a.x;
    my_deg = a.y;
    my_touch = P.g.lab[my_f] >> 31;
  }
  unsigned long long alg = 0, task_cnt = 0;  // warp-uniform

  // The chunk's candidates m are embeddings: position L holds each lane's w,
  // position pv (if any) each lane's cv, the others the stack.  Listing
  // reserves slots in the result table; a query past its listing budget
  // reserves none (its count stays exact, the host drops its partial tuples).
  auto emit = [&](uint32_t m, uint32_t w, uint32_t L, uint32_t pv, uint32_t cv) {
    uint32_t cnt = __popc(m);
    if (cnt == 0) return;
    task_cnt += cnt;
    if (!P.list) return;
    unsigned long long base = ~0ull;
    if (lane == 0) {
      bool ok = true;
      if (P.qlimit) ok = atomicAdd(&P.qlisted[Q.local], (unsigned long long)cnt) + cnt <= P.qlimit;
      if (ok) base = atomicAdd(&P.sc->out_count.v, (unsigned long long)cnt);
    }
    base = __shfl_sync(kFull, base, 0);
    if (base == ~0ull) return;
    alg += 4ull * (nq + 1) * cnt;  // the tuple and its segment id
    bool mine = (m >> lane) & 1u;
    unsigned long long s = base + __popc(m & lanemask_lt());
    bool wr = mine && s < P.cap;
    if (wr) P.out_seg[s] = seg;
    for (uint32_t k = 0; k < nq; ++k) {
      uint32_t pk = __shfl_sync(kFull, q_pos, k);
      uint32_t fk = __shfl_sync(kFull, my_f, pk & 31);
      if (wr) P.out_tup[s * P.W + k] = (pk == L) ? w : (pk == pv ? cv : fk);
    }
  };

  // Work limit (P.work_limit > 0): `work` counts the valid partial
  // embeddings of 3 or more positions this task generated (embeddings
  // included).  The total of a (query, update) segment does not depend on
  // scheduling, so "the segment's total reached the limit" is deterministic:
  // whoever's addition crosses it sets bit 63 of the segment's count, and the
  // segment's tasks stop (its count is then partial, marked by that bit).
  unsigned long long work = 0;
  auto publish_work = [&]() -> bool {  // true: the segment is over its limit
    uint32_t over = 0;
    if (lane == 0) {
      const unsigned long long before = work ? atomicAdd(&P.seg_work[seg], work) : ld_volatile(P.seg_work[seg]);
      over = before + work >= P.work_limit;
      if (work && before < P.work_limit && over) atomicOr(&P.seg_count[seg], kCountIncomplete);
    }
    work = 0;
    return __shfl_sync(kFull, over, 0) != 0;
  };

  auto flush = [&]() {
    if (P.work_limit && work) publish_work();
    if (lane == 0) {
      if (task_cnt) {
        atomicAdd(&P.seg_count[seg], task_cnt);
        atomicAdd(&P.sc->matches, task_cnt);
      }
      atomicAdd(&P.sc->alg_bytes, alg);
    }
  };

  if (depth >= nq) {  // a one-edge query: the seed is the embedding
    emit(1u, 0, 0xFFFFFFFFu, 0xFFFFFFFFu, 0);
    flush();
    return;
  }
  if (P.work_limit && publish_work()) return;  // a segment already over its limit

  const uint32_t pack_max = kLM ? P.pack_max : 0u;
  const uint32_t merge_max = kLM ? P.merge_max : 0u;
  // the current level (warp-uniform): its pivot run, next entry, end, pending
  // candidates of the last chunk, that chunk's first entry; its label and
  // backward neighbours
  uint32_t cur_base = 0, cur_pos = 0, cur_end = 0, cur_mask = 0, cur_chunk = 0, cur_pivot = 0;
  uint32_t cur_want = 0, cur_bn = 0;
  // level `lane`, parked while deeper levels run
  uint32_t lv_pos = 0, lv_end = 0, lv_mask = 0, lv_chunk = 0;

  // Level L scans the run of its pivot: the backward neighbour with the
  // fewest candidates (label-major: entries with L's label; plain: degree).
  // [rlo, rhi) narrows the scan for a donated range (rhi = 0: all of it).
  auto setup_level = [&](uint32_t L, uint32_t rlo, uint32_t rhi) {
    cur_bn = __shfl_sync(kFull, q_bn, L);
    cur_want = __shfl_sync(kFull, q_lab, L);
    const bool inb = (cur_bn >> lane) & 1u;
    uint32_t a = 0, b = my_deg;
    if constexpr (kLM) {
      b = 0;
      if (inb && cur_want < P.g.nlt) {
        const uint32_t *t = P.g.loff + (size_t)my_f * (P.g.nlt + 1) + cur_want;
        a = t[0];
        b = t[1];
      }
      // with packing, level nq - 2 also sets up the last level's ranges in
      // the runs of the positions before it (fixed while level nq - 2 runs)
      uint32_t fa = 0, fb = 0;
      bool fx = false;
      if (pack_max && L + 2 == nq) {
        const uint32_t bnn = __shfl_sync(kFull, q_bn, L + 1);
        const uint32_t wn = __shfl_sync(kFull, q_lab, L + 1);
        fx = lane < L && ((bnn >> lane) & 1u);
        if (fx && wn < P.g.nlt) {
          const uint32_t *t = P.g.loff + (size_t)my_f * (P.g.nlt + 1) + wn;
          fa = t[0];
          fb = t[1];
        }
        alg += 8ull * __popc(bnn & ((1u << L) - 1));
      }
      __syncwarp();  // lanes may still read these levels' previous ranges
      if (inb) srng[L][lane] = make_uint2(a, b);
      if (fx) srng[L + 1][lane] = make_uint2(fa, fb);
      if (pack_max && L + 2 == nq && lane == 0) stg->info = kStageUnset;  // a new context
      __syncwarp();
      alg += 8ull * __popc(cur_bn);
    }
    const uint32_t key = inb ? ((min(b - a, 0x3FFFFFFu) << 5) | lane) : 0xFFFFFFFFu;
    cur_pivot = __reduce_min_sync(kFull, key) & 31;
    cur_base = __shfl_sync(kFull, my_off, cur_pivot);
    const uint32_t pa = __shfl_sync(kFull, a, cur_pivot), pb = __shfl_sync(kFull, b, cur_pivot);
    cur_pos = rhi ? rlo : pa;
    cur_end = rhi ? min(rhi, pb) : pb;
    cur_mask = 0;
    cur_chunk = 0;
  };

  // The pivot of a level whose ranges are staged (label-major) or whose
  // backward neighbours' degrees are at hand (plain): the same choice
  // setup_level made, recomputed instead of parked.
  auto pivot_of = [&](uint32_t L) -> uint32_t {
    const uint32_t bnL = __shfl_sync(kFull, q_bn, L);
    const bool inb = (bnL >> lane) & 1u;
    uint32_t len = my_deg;
    if constexpr (kLM) {
      const uint2 r = inb ? srng[L][lane] : make_uint2(0, 0);
      len = r.y - r.x;
    }
    const uint32_t key = inb ? ((min(len, 0x3FFFFFFu) << 5) | lane) : 0xFFFFFFFFu;
    return __reduce_min_sync(kFull, key) & 31;
  };
  auto pivot_base = [&](uint32_t L) -> uint32_t { return __shfl_sync(kFull, my_off, pivot_of(L)); };
  auto resume_pivot = [&](uint32_t L) {
    cur_pivot = pivot_of(L);
    cur_base = __shfl_sync(kFull, my_off, cur_pivot);
  };

  uint32_t hb = 0;  // chunks since the last heartbeat

  // The packed last level over the candidates m of level L = nq - 2 (lane k:
  // candidate cw, its label word clw).  False: more than pack_max entries (or
  // one range longer than that), nothing done.
  auto pack_last = [&](uint32_t L, uint32_t m, uint32_t cw, uint32_t clw) -> bool {
    const uint32_t LL = L + 1;
    const uint32_t bnn = __shfl_sync(kFull, q_bn, LL);
    const uint32_t wn = __shfl_sync(kFull, q_lab, LL);
    const bool dep = (bnn >> L) & 1u;  // the last level reads the candidate's own run
    const uint32_t fixed = bnn & ~(1u << L);
    uint2 fr = make_uint2(0, 0);
    uint32_t fkey = 0xFFFFFFFFu;
    if ((fixed >> lane) & 1u) {
      fr = srng[LL][lane];
      fkey = (min(fr.y - fr.x, 0x3FFFFFFu) << 5) | lane;
    }
    const uint32_t fmin = __reduce_min_sync(kFull, fkey);
    const uint32_t fj = fmin & 31;  // the shortest fixed range (none: fmin = ~0)
    const uint32_t f_off = __shfl_sync(kFull, my_off, fj);
    const uint32_t f_a = __shfl_sync(kFull, fr.x, fj);
    const uint32_t f_b = __shfl_sync(kFull, fr.y, fj);
    const uint32_t f_len = fmin == 0xFFFFFFFFu ? 0xFFFFFFFFu : f_b - f_a;
    const bool cand = (m >> lane) & 1u;
    uint32_t o_off = 0, o_a = 0, o_b = 0;
    if (cand && dep && wn < P.g.nlt) {
      o_off = P.g.adj[cw].x;
      const uint32_t *t = P.g.loff + (size_t)cw * (P.g.nlt + 1) + wn;
      o_a = t[0];
      o_b = t[1];
    }
    const bool own = dep && (o_b - o_a) < f_len;
    const uint32_t len = cand ? (own ? o_b - o_a : f_len) : 0u;
    if (__any_sync(kFull, len > pack_max)) return false;
    uint32_t incl = len;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += t;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    if (total > pack_max) return false;
    if (dep) alg += 8ull * __popc(m);
    // candidate k's entry, read by the lanes whose entries fall in its range
    __syncwarp();  // the previous pass's lanes may still read the table
    spk[lane] = PackEnt{incl - len, cw, o_off, o_a, o_b, (own ? 1u : 0u) | ((clw >> 31) << 1), 0u, 0u};
    uint32_t sinfo = stg->info;
    __syncwarp();
    if (sinfo == kStageUnset) {  // first pass of this context: stage the longest fixed range
      const uint32_t lkey = ((fixed >> lane) & 1u) ? ((min(fr.y - fr.x, 0x3FFFFFFu) << 5) | lane) : 0u;
      const uint32_t lmax = __reduce_max_sync(kFull, lkey);
      const uint32_t slen = lmax >> 5, sj = lmax & 31;
      sinfo = kStageNone;
      if (slen >= kStageMin) {
        uint32_t shift = 0;
        while ((slen >> shift) > kStage) ++shift;
        const uint32_t nf = (slen + (1u << shift) - 1) >> shift;
        const uint32_t *src = P.g.arena + (uint64_t)__shfl_sync(kFull, my_off, sj) * 4 + __shfl_sync(kFull, fr.x, sj);
        for (uint32_t i = lane; i < nf; i += 32) stg->fence[i] = src[(size_t)i << shift];
        alg += 4ull * nf;
        sinfo = sj | (shift << 5) | (nf << 10);
      }
      if (lane == 0) stg->info = sinfo;
      __syncwarp();
    }
    const uint32_t st_j = sinfo < kStageNone ? (sinfo & 31) : 32u;
    const uint32_t same = __ballot_sync(kFull, lane < L && q_lab == wn);
    const bool sameP = cur_want == wn;
    const uint32_t qvn = __shfl_sync(kFull, q_vert, LL);
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t t = base + lane;
      bool ok = t < total;
      // the candidate whose range holds entry t: the first lane with incl > t
      uint32_t k = 0;
#pragma unroll
      for (uint32_t s = 16; s; s >>= 1) {
        const uint32_t v = __shfl_sync(kFull, incl, k + s - 1);
        if (v <= t) k += s;
      }
      const PackEnt pe = spk[k];
      const uint32_t kx = pe.excl, kc = pe.cw, ko = pe.off, ka = pe.a, kb = pe.b, kf = pe.flags;
      const bool kown = kf & 1u;
      const uint64_t start = kown ? (uint64_t)ko * 4 + ka : (uint64_t)f_off * 4 + f_a;
      const uint32_t e = ok ? P.g.arena[start + (t - kx)] : 0u;
      const uint32_t w = e & kIdMask;
      uint32_t lw = 0;
      if (wn >= 31) {  // slot 31 holds every label >= 31
        lw = ok ? P.g.lab[w] : 0u;
        ok = ok && ((lw & kLabelMask) == wn);
      }
      for (uint32_t sm = same; sm; sm &= sm - 1) {
        const uint32_t fjv = __shfl_sync(kFull, my_f, __ffs(sm) - 1);
        ok = ok && (w != fjv);
      }
      if (sameP) ok = ok && (w != kc);
      if (bitmap) ok = ok && ((bitmap[(size_t)qvn * col_len + (w >> 5)] >> (w & 31)) & 1u);
      uint32_t probes = 0;
      for (uint32_t bits = bnn; bits; bits &= bits - 1) {
        const uint32_t j = __ffs(bits) - 1;
        const uint32_t oj = __shfl_sync(kFull, my_off, j);
        const bool piv = kown ? (j == L) : (j == fj);
        if (ok && !piv) {
          uint32_t ra, rb;
          const uint32_t *lst;
          if (j == L) {
            lst = P.g.arena + (uint64_t)ko * 4;
            ra = ka;
            rb = kb;
          } else {
            const uint2 r = srng[LL][j];
            lst = P.g.arena + (uint64_t)oj * 4;
            ra = r.x;
            rb = r.y;
          }
          if (j == st_j) {
            // fences in shared memory: lo = first fence >= e; a miss there
            // leaves the window between fences lo - 1 and lo in global memory
            const uint32_t shift = (sinfo >> 5) & 31, nf = sinfo >> 10;
            const uint32_t lo = lower_bound_u32(stg->fence, nf, e);
            if (lo < nf && stg->fence[lo] == e) {
              ok = true;
            } else if (lo == 0 || shift == 0) {
              ok = false;
            } else {
              const uint32_t wa = ra + ((lo - 1) << shift) + 1, wb = min(ra + (lo << shift), rb);
              const uint32_t p = wa + lower_bound_u32(lst + wa, wb - wa, e);
              ok = p < wb && lst[p] == e;
            }
          } else {
            const uint32_t p = ra + lower_bound_u32(lst + ra, rb - ra, e);
            ok = p < rb && lst[p] == e;
          }
          ++probes;
        }
      }
      if (wn < 31) lw = ok ? P.g.lab[w] : 0u;  // touch bit of the survivors
      if (__any_sync(kFull, ok && (lw >> 31))) {
        for (uint32_t bits = bnn; bits; bits &= bits - 1) {
          const uint32_t j = __ffs(bits) - 1;
          uint32_t fjv = __shfl_sync(kFull, my_f, j), tj = __shfl_sync(kFull, my_touch, j);
          if (j == L) {
            fjv = kc;
            tj = (kf >> 1) & 1u;
          }
          if (ok && (lw >> 31) && tj) ok = edge_live(bt, fjv, w, tp);
        }
      }
      const uint32_t m2 = __ballot_sync(kFull, ok);
      work += __popc(m2);
      alg += 4ull * min(32u, total - base) + 4ull * __reduce_add_sync(kFull, probes);
      emit(m2, w, LL, L, kc);
      ++hb;
    }
    return true;
  };

  // Breadth-first rows: the candidates m of level L (lane k: cw) become
  // rows of L + 1 fixed positions.  One reservation per chunk, all or
  // nothing (a bounded compare-and-swap loop); false: no room, nothing
  // written.
  auto write_rows = [&](uint32_t L, uint32_t m, uint32_t cw) -> bool {
    const uint32_t cnt = __popc(m);
    unsigned long long base = ~0ull;
    if (lane == 0) {
      unsigned long long cur = ld_volatile(*P.rows_cnt);
      for (int tries = 0; tries < 64 && cur + cnt <= P.rows_cap; ++tries) {
        const unsigned long long prev = atomicCAS(P.rows_cnt, cur, cur + cnt);
        if (prev == cur) {
          base = cur;
          break;
        }
        cur = prev;
      }
    }
    base = __shfl_sync(kFull, base, 0);
    if (base == ~0ull) return false;
    const uint32_t fsrc = __shfl_sync(kFull, my_f, (lane - 8) & 31);
    uint32_t bits = m;
    for (uint32_t r = 0; r < cnt; ++r) {
      const uint32_t b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t cb = __shfl_sync(kFull, cw, b);
      uint32_t word = 0;
      if (lane == 0) word = upd;
      else if (lane == 1) word = qo;
      else if (lane == 2) word = L + 1;
      else if (lane >= 8 && lane < 24) {
        const uint32_t fi = lane - 8;
        word = fi < L ? fsrc : (fi == L ? cb : 0u);
      }
      __stcg(reinterpret_cast<uint32_t *>(P.rows_out + base + r) + lane, word);
    }
    return true;
  };

  uint32_t L = depth;
  setup_level(L, lo, hi);
  uint32_t dticks = 0;  // chunks since the last donation check
  while (true) {
    if (cur_mask == 0) {
      if (cur_pos >= cur_end) {
        if (L == depth) break;
        --L;  // back to the parked level
        cur_pos = __shfl_sync(kFull, lv_pos, L);
        cur_end = __shfl_sync(kFull, lv_end, L);
        cur_mask = __shfl_sync(kFull, lv_mask, L);
        cur_chunk = __shfl_sync(kFull, lv_chunk, L);
        cur_bn = __shfl_sync(kFull, q_bn, L);
        cur_want = __shfl_sync(kFull, q_lab, L);
        resume_pivot(L);
        continue;
      }
      const uint32_t pos = cur_pos, end = cur_end;
      const uint32_t *run = P.g.arena + (uint64_t)cur_base * 4;
      const uint32_t i = pos + lane;
      bool ok = i < end;
      const uint32_t e = ok ? run[i] : 0;  // entry (label-major) or id
      const uint32_t w = kLM ? (e & kIdMask) : e;
      const uint32_t want = cur_want;
      uint32_t lw = 0;
      if constexpr (kLM) {
        if (want >= 31) {  // slot 31 holds every label >= 31
          lw = ok ? P.g.lab[w] : 0;
          ok = ok && ((lw & kLabelMask) == want);
        }
      } else {
        lw = ok ? P.g.lab[w] : 0;
        ok = ok && ((lw & kLabelMask) == want);
      }
      // injectivity: only earlier positions with the same label can hold w
      for (uint32_t same = __ballot_sync(kFull, lane < L && q_lab == want); same; same &= same - 1) {
        const uint32_t fj = __shfl_sync(kFull, my_f, __ffs(same) - 1);
        ok = ok && (w != fj);
      }
      if (bitmap) {
        const uint32_t qv = __shfl_sync(kFull, q_vert, L);
        ok = ok && ((bitmap[(size_t)qv * col_len + (w >> 5)] >> (w & 31)) & 1u);
      }
      const uint32_t bnL = cur_bn;
      uint32_t others = bnL & ~(1u << cur_pivot);
      uint32_t probes = 0;
      while (others) {
        uint32_t j = __ffs(others) - 1;
        others &= others - 1;
        const uint32_t oj = __shfl_sync(kFull, my_off, j);
        if constexpr (kLM) {
          const uint2 r = srng[L][j];
          const uint32_t *lst = P.g.arena + (uint64_t)oj * 4;
          const uint32_t nb = r.y - r.x;
          if (nb <= merge_max) {
            // merge: the chunk's entries (ascending across lanes) against
            // the range in 32-entry tiles, each lane placing its entry in a
            // tile by a five-step shuffle search; stops at the first tile
            // that reaches the chunk's largest live entry
            const uint32_t emax = __reduce_max_sync(kFull, ok ? e : 0u);
            bool found = false;
            for (uint32_t t = 0; t < nb; t += 32) {
              const uint32_t bv = t + lane < nb ? lst[r.x + t + lane] : 0xFFFFFFFFu;
              uint32_t k = 0;
#pragma unroll
              for (uint32_t sh = 16; sh; sh >>= 1)
                if (__shfl_sync(kFull, bv, k + sh - 1) < e) k += sh;
              const uint32_t at = __shfl_sync(kFull, bv, k);  // every lane shuffles
              const uint32_t last = __shfl_sync(kFull, bv, 31);
              if (at == e && t + k < nb) found = true;
              if (last >= emax) break;
            }
            probes += ok ? 1u : 0u;
            ok = ok && found;
          } else if (ok) {
            const uint32_t p = r.x + lower_bound_u32(lst + r.x, nb, e);
            ok = p < r.y && lst[p] == e;
            ++probes;
          }
        } else {
          const uint32_t dj = __shfl_sync(kFull, my_deg, j);
          if (ok) {
            const uint32_t *lst = P.g.arena + (uint64_t)oj * 4;
            uint32_t p = lower_bound_u32(lst, dj, w);
            ok = p < dj && lst[p] == w;
            ++probes;
          }
        }
      }
      if constexpr (kLM) {
        if (want < 31) lw = ok ? P.g.lab[w] : 0;  // touch bit of the survivors
      }
      if (__any_sync(kFull, ok && (lw >> 31))) {
        uint32_t bits = bnL;
        while (bits) {
          uint32_t j = __ffs(bits) - 1;
          bits &= bits - 1;
          uint32_t fj = __shfl_sync(kFull, my_f, j), tj = __shfl_sync(kFull, my_touch, j);
          if (ok && (lw >> 31) && tj) ok = edge_live(bt, fj, w, tp);
        }
      }
      const uint32_t m = __ballot_sync(kFull, ok);
      work += __popc(m);
      alg += (kLM ? 4ull : 8ull) * min(32u, end - pos) + 4ull * __reduce_add_sync(kFull, probes);
      cur_pos = pos + 32;
      cur_chunk = pos;
      ++hb;
      ++dticks;
      if (L == nq - 1) {
        emit(m, w, L, 0xFFFFFFFFu, 0);
      } else if (kLM && pack_max && L + 2 == nq && m) {
        if (!pack_last(L, m, w, lw)) cur_mask = m;
      } else if (P.bfs_stop == L + 1 && m) {
        if (!write_rows(L, m, w)) cur_mask = m;
      } else {
        cur_mask = m;
      }

      if (hb >= 64) {
        hb = 0;
        unsigned int err = 0;
        if (lane == 0) {
          atomicAdd(&P.sc->progress.v, 1ull);
          err = ld_volatile(P.sc->error);
        }
        if (__shfl_sync(kFull, err, 0)) break;
        if (P.work_limit && publish_work()) break;
      }
      if (P.donate && dticks >= 8) {
        dticks = 0;
        const uint32_t split_min = P.split_min > 64 ? P.split_min : (P.split_min ? 64u : 128u);
        const uint32_t dd = P.donate_depth ? min(P.donate_depth, 4u) : 2u;
        unsigned long long h = 0;
        if (lane == 0) {
          unsigned long long pc = ld_volatile(P.sc->pop_cnt.v), pu = ld_volatile(P.sc->push_cnt.v);
          h = pc > pu ? pc - pu : 0;
        }
        h = __shfl_sync(kFull, h, 0);
        if (h > 0) {
          if (lane == L) {  // park the current level, so every level reads alike
            lv_pos = cur_pos;
            lv_end = cur_end;
            lv_mask = cur_mask;
            lv_chunk = cur_chunk;
          }
          // shallowest level with a substantial piece of work: pending
          // candidates with dd or more levels below them, or a remaining
          // range of split_min entries or more
          bool has = lane >= depth && lane <= L &&
                     ((lv_mask != 0 && lane + dd < nq) || lv_end >= lv_pos + split_min);
          uint32_t hm = __ballot_sync(kFull, has);
          if (hm) {
            const uint32_t p = __ffs(hm) - 1;
            const uint32_t pm0 = __shfl_sync(kFull, lv_mask, p);
            const uint32_t pm = (p + dd < nq) ? pm0 : 0u;
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
            const unsigned long long rmask = P.job_ring - 1;
            if (lane == 0) {
              // k <= waiting warps, so positions stay within one warp's worth
              // of reservations per donor of pop_cnt: the slot of position p
              // was last used by position p - ring, consumed long ago; wait
              // (bounded) until its consumer has released it
              atomicAdd(&P.sc->outstanding.v, (unsigned long long)k);
              s0 = atomicAdd(&P.sc->push_cnt.v, (unsigned long long)k);
              atomicAdd(&P.sc->donations, (unsigned long long)k);
              okr = 1;
              long long tw = clock64();
              for (uint32_t r = 0; r < k && okr; ++r)
                while (ld_volatile(P.job_seq[(s0 + r) & rmask]) != s0 + r) {
                  if (clock64() - tw > P.timeout_cycles) {
                    atomicOr(&P.sc->error, kErrTimeout);
                    okr = 0;
                    break;
                  }
                  __nanosleep(64);
                }
            }
            okr = __shfl_sync(kFull, okr, 0);
            s0 = __shfl_sync(kFull, s0, 0);
            if (okr) {
              // level p's pivot run (its ranges are still staged)
              const uint32_t pbase = pivot_base(p);
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
                  if constexpr (kLM) cw &= kIdMask;
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
                uint32_t *rec = reinterpret_cast<uint32_t *>(P.jobs + ((s0 + r) & rmask));
                __stcg(rec + lane, word);
              }
              __threadfence();
              __syncwarp();
              if (lane < k) atomicExch(&P.job_seq[(s0 + lane) & rmask], s0 + lane + 1);
              if (lane == p) {
                if (pm) lv_mask &= ~dmask;
                else lv_end = rmid;
              }
              if (p == L) {  // the donated piece came from the current level
                if (pm) cur_mask &= ~dmask;
                else cur_end = rmid;
              }
            }
          }
        }
      }
      continue;
    }
    // descend into the lowest pending candidate of level L
    const uint32_t b = __ffs(cur_mask) - 1;
    uint32_t w = P.g.arena[(uint64_t)cur_base * 4 + cur_chunk + b];
    if constexpr (kLM) w &= kIdMask;
    cur_mask &= cur_mask - 1;
    if (lane == L) {
      lv_pos = cur_pos;
      lv_end = cur_end;
      lv_mask = cur_mask;
      lv_chunk = cur_chunk;
      my_f = w;
      uint2 a = P.g.adj[w];
      my_off = a.x;
      my_deg = a.y;
      my_touch = P.g.lab[w] >> 31;
    }
    ++L;
    setup_level(L, 0, 0);
  }
  flush();
}

// phantom = 1 adds one outstanding task that nothing finishes (a test of the
// bounded waits: the launch then ends only through their timeouts).
__global__ void k_sched_init(Sched *sc, const BatchHdr *hdr, unsigned long long *job_seq, uint32_t job_ring,
                             uint32_t phantom) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long seed_cap = hdr ? hdr->seed_cap : ~0ull;  // no header: tasks are rows
  for (uint32_t s = i; s < job_ring; s += gridDim.x * blockDim.x) job_seq[s] = s;
  if (i == 0) {
    unsigned long long n = sc->nseeds;
    if (n > seed_cap) {
      sc->nseeds = n = seed_cap;
      atomicOr(&sc->error, kErrSeeds);
    }
    sc->outstanding.v = n + phantom;
    sc->done.v = (n + phantom == 0) ? 1ull : 0ull;
  }
}

// kMinBlocks: resident blocks per SM the register allocation is sized for
// (5: 48 registers a thread; 4: 64).  Launches of 5 or more blocks per SM
// take the first, fewer the second.
template <bool kLM, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) k_match(MatchArgs P) {
  __shared__ uint2 s_rng[kLM ? 8 : 1][16][16];
  __shared__ PackEnt s_pack[kLM ? 8 : 1][32];
  __shared__ PackStage s_stage[kLM ? 8 : 1];
  const uint32_t lane = threadIdx.x & 31;
  if (*P.abort_flag & kErrArena) return;  // the batch was refused before its insert
  // an earlier launch of this batch failed (one read, the same for the warp:
  // the word can change while the kernel runs)
  if (__shfl_sync(kFull, lane == 0 ? ld_volatile(P.sc->error) : 0u, 0)) return;
  const uint32_t nupd = P.hdr->n;
  const DevBatchEdges bt{P.bt.bkey, P.bt.binfo, P.hdr->m};
  bool seeds_done = false;
  while (true) {
    uint32_t kind = 0;
    unsigned long long slot = 0;
    if (lane == 0) kind = acquire(P, slot, seeds_done);
    kind = __shfl_sync(kFull, kind, 0);
    if (kind == 0) break;
    slot = __shfl_sync(kFull, slot, 0);
    uint32_t upd, qo, depth, lo = 0, hi = 0, fval = 0;
    if (kind == 1 && P.rows_in) {  // a row written by the previous launch
      const uint32_t word = __ldcg(reinterpret_cast<const uint32_t *>(P.rows_in + slot) + lane);
      upd = __shfl_sync(kFull, word, 0);
      qo = __shfl_sync(kFull, word, 1);
      depth = __shfl_sync(kFull, word, 2);
      fval = __shfl_sync(kFull, word, (lane + 8) & 31);
    } else if (kind == 1) {
      uint4 s = P.seeds[slot];
      upd = s.x;
      qo = s.y;
      depth = 2;
      fval = lane == 0 ? s.z : (lane == 1 ? s.w : 0u);
    } else {
      const uint32_t *rec = reinterpret_cast<const uint32_t *>(P.jobs + (slot & (P.job_ring - 1)));
      uint32_t word = __ldcg(rec + lane);
      __syncwarp();
      if (lane == 0) {  // the slot is free for position slot + ring
        __threadfence();
        atomicExch(&P.job_seq[slot & (P.job_ring - 1)], slot + P.job_ring);
      }
      upd = __shfl_sync(kFull, word, 0);
      qo = __shfl_sync(kFull, word, 1);
      depth = __shfl_sync(kFull, word, 2);
      lo = __shfl_sync(kFull, word, 3);
      hi = __shfl_sync(kFull, word, 4);
      fval = __shfl_sync(kFull, word, (lane + 8) & 31);
    }
    run_task<kLM>(P, bt, nupd, upd, qo, depth, lo, hi, fval, s_rng[kLM ? (threadIdx.x >> 5) : 0],
                  s_pack[kLM ? (threadIdx.x >> 5) : 0], &s_stage[kLM ? (threadIdx.x >> 5) : 0]);
    finish_task(P);
  }
}

}  // namespace

__global__ void k_rows_arm(Sched *sc, const unsigned long long *rows_cnt, unsigned long long rows_cap) {
  sc->seeds = sc->nseeds;  // the seed table's count, for a rerun from the seeds
  sc->seed_next.v = 0;
  sc->push_cnt.v = 0;
  sc->pop_cnt.v = 0;
  sc->done.v = 0;
  sc->outstanding.v = 0;
  sc->nseeds = min(*rows_cnt, rows_cap);
}

void launch_rows_arm(Sched *sc, const unsigned long long *rows_cnt, unsigned long long rows_cap, cudaStream_t s) {
  k_rows_arm<<<1, 1, 0, s>>>(sc, rows_cnt, rows_cap);
}

void launch_sched_init(Sched *sc, const BatchHdr *hdr, unsigned long long *job_seq, uint32_t job_ring,
                       cudaStream_t s, uint32_t phantom) {
  k_sched_init<<<(job_ring + 255) / 256, 256, 0, s>>>(sc, hdr, job_seq, job_ring, phantom);
}

void launch_match(const MatchArgs &a, int blocks, cudaStream_t s) {
  int dev = 0, sms = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool wide = blocks < 5 * std::max(sms, 1);  // fewer than 5 blocks per SM: 64 registers
  if (!a.g.loff) k_match<false, 5><<<blocks, 256, 0, s>>>(a);
  else if (wide) k_match<true, 4><<<blocks, 256, 0, s>>>(a);
  else k_match<true, 5><<<blocks, 256, 0, s>>>(a);
}

int match_max_blocks_per_sm() {
  int n = 0, m = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_match<true, 5>, 256, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_match<false, 5>, 256, 0);
  return n < m ? n : m;
}

}  // namespace dsm
