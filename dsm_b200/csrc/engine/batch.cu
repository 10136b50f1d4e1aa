// The batch pipeline of the engine: one device batch = one iteration of the
// reference's loop (main.cu:152-347: updateHostGraph, re-upload, re-filter,
// seeding, matching) for every registered query at once.
//
//   prepare        host only: canonical keys (sorted), directed pairs grouped
//                  by source vertex, all in the slot's pinned staging buffer
//   launch_front   uploads; segment A = clear, edge state, arena check, union
//                  insert, filters, seeds, scheduler, matcher, read-back of
//                  the scheduler (one executable CUDA graph, replayed while
//                  its buffers and settings stay the same: the kernels read
//                  the batch's sizes from a device header)
//   finish_device  waits for the matcher; regrows the result table and
//                  reruns on overflow; segment B = deletions and marks; the
//                  downloads into the slot's pinned buffers
//   assemble       waits for the downloads; per-(query, update) counts and
//                  canonically sorted tuples
//
// An arena that cannot hold the batch's relocated runs is detected on the
// device before anything is written: the insert, the matcher and the deletes
// then skip, the batch leaves the graph as it was, and the engine compacts
// the arena (growing it within the budget) and runs the batch again.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/dsm.h"
#include "../host/par.h"
#include "engine_internal.h"
#include "filter.cuh"
#include "kernels.cuh"

namespace dsm {

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace {

constexpr int kRetryArena = -100;  // internal: compact the arena and run the batch again

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

template <class T>
void key_append(std::string &k, const T &x) {
  k.append(reinterpret_cast<const char *>(&x), sizeof(T));
}

}  // namespace

// ---------------------------------------------------------------------------
// host preparation
// ---------------------------------------------------------------------------
int Engine::prepare(const dsm_update *ups, uint32_t n, Staged &S, int slot) {
  const auto t0 = std::chrono::steady_clock::now();
  S = Staged();
  S.ups = ups;
  S.n = n;
  S.slot = slot;
  HostOut &H = hout[slot];
  std::vector<std::pair<uint64_t, uint32_t>> und;
  und.reserve(n);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t a = ups[i].src, b = ups[i].dst;
    if (a == b) continue;
    und.push_back({a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a, i});
  }
  std::sort(und.begin(), und.end());
  S.m = (uint32_t)und.size();
  std::vector<uint64_t> dir;
  dir.reserve(2 * (size_t)S.m);
  for (auto &e : und) {  // x << 32 | entry of y, so each group is in run order
    const uint32_t a = (uint32_t)(e.first >> 32), b = (uint32_t)e.first;
    dir.push_back(((uint64_t)a << 32) | entry_of(b));
    dir.push_back(((uint64_t)b << 32) | entry_of(a));
  }
  std::sort(dir.begin(), dir.end());
  std::vector<uint32_t> dhead;
  for (size_t j = 0; j < dir.size(); ++j)
    if (j == 0 || (dir[j] >> 32) != (dir[j - 1] >> 32)) dhead.push_back((uint32_t)j);
  S.ngroups = (uint32_t)dhead.size();
  dhead.push_back((uint32_t)dir.size());
  S.ndir = dir.size();
  const size_t up_bytes = (size_t)n * 16, bk_bytes = (size_t)S.m * 8, bi_bytes = (size_t)S.m * 4,
               dk_bytes = dir.size() * 8, dh_bytes = dhead.size() * 4;
  S.o_up = 0;
  S.o_bk = up_bytes;
  S.o_bi = S.o_bk + bk_bytes;
  S.o_dk = (S.o_bi + bi_bytes + 7) & ~(size_t)7;
  S.o_dh = S.o_dk + dk_bytes;
  if (int rc = halloc(H.stage, S.o_dh + dh_bytes + 64)) return rc;
  char *st = (char *)H.stage.ptr;
  std::memcpy(st + S.o_up, ups, up_bytes);
  for (uint32_t j = 0; j < S.m; ++j) {
    ((uint64_t *)(st + S.o_bk))[j] = und[j].first;
    ((uint32_t *)(st + S.o_bi))[j] = und[j].second;
  }
  std::memcpy(st + S.o_dk, dir.data(), dk_bytes);
  std::memcpy(st + S.o_dh, dhead.data(), dh_bytes);
  S.host_prep_ms = ms_since(t0);
  return DSM_OK;
}

// ---------------------------------------------------------------------------
// device segments
// ---------------------------------------------------------------------------
int Engine::seg_a_kernels(Staged &S, const ClearArgs &ca, const EdgeStateArgs &es, const AdjUpdateArgs &au,
                          const SeedArgs &sa, bool seeds) {
  const int blocks = num_sms * 4;
  launch_batch_clear(ca, blocks, stream);
  launch_edge_state(es, blocks, stream);
  launch_arena_check(au, blocks, stream);
  launch_adj_insert(au, blocks, stream);
  if (int r = rec(ev_pool[1])) return r;
  stats.kernel_launches += 4;
  if (S.match) {
    if (int r = launch_filters()) return r;  // per query, on the union graph
    if (seeds) {
      launch_seeds(sa, blocks, stream);
      launch_sched_init((Sched *)d_sched.ptr, (const BatchHdr *)d_hdr.ptr, (unsigned long long *)d_job_seq.ptr,
                        job_ring, stream, stall_test);
      stats.kernel_launches += 2;
    }
  }
  return DSM_OK;
}

int Engine::launch_front(Staged &S) {
  if (int rc = sync_queries()) return rc;
  HostOut &H = hout[S.slot];
  const uint32_t n = S.n, m = S.m;
  S.nq_live = (uint32_t)live_ids.size();
  S.qids = live_ids;
  S.widths.clear();
  for (uint32_t id : live_ids) S.widths.push_back(slots[id].plan.nq);
  S.W = std::max<uint32_t>(max_width, 1);
  S.plain = plain;
  S.sort = sort_results;
  S.qlimit = list_mode ? query_list_limit : 0;
  if (S.nq_live == 0) S.match = false;
  const size_t nn = std::max<uint32_t>(n, 1), mm = std::max<uint32_t>(m, 1), dd = std::max<size_t>(S.ndir, 1);
  S.seed_cap = (unsigned long long)nn * std::max<uint32_t>(max_bucket, 1);
  S.nseg = (size_t)std::max<uint32_t>(S.nq_live, 1) * nn;
  int rc;
  if ((rc = dalloc(d_upd, nn * 16)) || (rc = dalloc(d_bkey, mm * 8)) || (rc = dalloc(d_bidx, mm * 4)) ||
      (rc = dalloc(d_binfo, mm * 4)) || (rc = dalloc(d_gflag, mm)) || (rc = dalloc(d_vtp, nn * 4)) ||
      (rc = dalloc(d_dkey, dd * 8)) || (rc = dalloc(d_dhead, (dd + 1) * 4)) || (rc = dalloc(d_dsel, dd * 4)) ||
      (rc = dalloc(d_segcnt, S.nseg * 8)) || (rc = dalloc(d_qlisted, std::max<size_t>(S.nq_live, 1) * 8)))
    return rc;
  S.work_limit = S.match ? work_limit : 0;
  if (S.work_limit && (rc = dalloc(d_segwork, S.nseg * 8))) return rc;
  if (S.match && (rc = dalloc(d_seeds, S.seed_cap * 16))) return rc;
  if (S.match && (bfs_levels || (tune_next && !S.plain)) && (rc = dalloc(d_rows, bfs_rows * sizeof(JobRec))))
    return rc;
  if (!d_jobs.ptr) {
    if ((rc = dalloc(d_jobs, (size_t)job_ring * sizeof(JobRec))) || (rc = dalloc(d_job_seq, (size_t)job_ring * 8)))
      return rc;
  }
  if (list_mode && S.match) {
    const size_t cap = std::max<uint64_t>(result_cap, 1024);
    if ((rc = dalloc(d_out_seg, cap * 4)) || (rc = dalloc(d_out_tup, cap * S.W * 4))) return rc;
  }
  // what allocates, synchronises or copies pageable memory runs before the
  // segments, so that each segment can be captured into a CUDA graph
  if (!(S.match && filter_mode > 0) && d_rinfo.ptr && n)  // the graph changes unfiltered
    CK(cudaMemsetAsync(d_rinfo.ptr, 1, 1, stream));  // RegionInfo::stale
  if (qd_dirty)
    if ((rc = upload_qd())) return rc;
  if (S.match && (rc = prepare_filters())) return rc;
  if ((rc = halloc(H.segcnt, S.nseg * 8)) || (rc = halloc(H.vtp, nn * 4)) || (rc = halloc(H.misc, 256)) ||
      (rc = halloc(H.hdr, sizeof(BatchHdr))) || (rc = halloc(h_qlisted, std::max<size_t>(S.nq_live, 1) * 8)))
    return rc;
  if (!H.ev0) {
    CK(cudaEventCreate(&H.ev0));
    CK(cudaEventCreate(&H.ev_end));
  }
  BatchHdr &hd = *(BatchHdr *)H.hdr.ptr;
  hd.n = n;
  hd.m = m;
  hd.ngroups = S.ngroups;
  hd.nq_live = S.nq_live;
  hd.seed_cap = S.seed_cap;
  hd.nseg = (unsigned long long)S.nq_live * n;

  // uploads (plain copies from the slot's pinned staging)
  CK(cudaEventRecord(H.ev0, stream));
  const char *st = (const char *)H.stage.ptr;
  CK(cudaMemcpyAsync(d_hdr.ptr, H.hdr.ptr, sizeof(BatchHdr), cudaMemcpyHostToDevice, stream));
  if (n) CK(cudaMemcpyAsync(d_upd.ptr, st + S.o_up, (size_t)n * 16, cudaMemcpyHostToDevice, stream));
  if (m) {
    CK(cudaMemcpyAsync(d_bkey.ptr, st + S.o_bk, (size_t)m * 8, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d_bidx.ptr, st + S.o_bi, (size_t)m * 4, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d_dkey.ptr, st + S.o_dk, S.ndir * 8, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d_dhead.ptr, st + S.o_dh, (S.ngroups + 1) * 4, cudaMemcpyHostToDevice, stream));
  }

  DevGraph g = dev_graph();
  const BatchHdr *dh = (const BatchHdr *)d_hdr.ptr;
  unsigned int *d_err = (unsigned int *)d_misc.ptr;
  unsigned long long *segwork = S.work_limit ? (unsigned long long *)d_segwork.ptr : nullptr;
  ClearArgs ca{dh, (uint32_t *)d_vtp.ptr, (unsigned long long *)d_segcnt.ptr, segwork,
               (unsigned long long *)d_qlisted.ptr, (Sched *)d_sched.ptr, (uint32_t *)d_misc.ptr};
  EdgeStateArgs es{g, dh, (const uint4 *)d_upd.ptr, (const unsigned long long *)d_bkey.ptr,
                   (const uint32_t *)d_bidx.ptr, (uint32_t *)d_binfo.ptr, (uint8_t *)d_gflag.ptr,
                   (uint32_t *)d_vtp.ptr};
  AdjUpdateArgs au{g, dh, (const unsigned long long *)d_dkey.ptr, (const uint32_t *)d_dhead.ptr,
                   (const unsigned long long *)d_bkey.ptr, (const uint8_t *)d_gflag.ptr, (uint32_t *)d_dsel.ptr,
                   d_err, (unsigned long long *)((char *)d_misc.ptr + 8),
                   (unsigned long long *)((char *)d_misc.ptr + 16)};
  SeedArgs sa{g, dh, (const uint4 *)d_upd.ptr, (const uint32_t *)d_vtp.ptr, (const uint32_t *)d_pair_off.ptr,
              (const uint32_t *)d_pair_ent.ptr, (const QDev *)d_qd.ptr, (const OrderRec *)d_orders.ptr,
              (uint4 *)d_seeds.ptr, (Sched *)d_sched.ptr, kAllSlots};
  MatchArgs ma;
  std::memset(&ma, 0, sizeof(ma));
  ma.g = g;
  ma.bt = DevBatchEdges{(const unsigned long long *)d_bkey.ptr, (const uint32_t *)d_binfo.ptr, 0};
  ma.hdr = dh;
  ma.vtp = (const uint32_t *)d_vtp.ptr;
  ma.qd = (const QDev *)d_qd.ptr;
  ma.orders = (const OrderRec *)d_orders.ptr;
  ma.seeds = (const uint4 *)d_seeds.ptr;
  ma.sc = (Sched *)d_sched.ptr;
  ma.jobs = (JobRec *)d_jobs.ptr;
  ma.job_seq = (unsigned long long *)d_job_seq.ptr;
  ma.job_ring = job_ring;
  ma.W = S.W;
  ma.seg_count = (unsigned long long *)d_segcnt.ptr;
  ma.qlisted = (unsigned long long *)d_qlisted.ptr;
  ma.qlimit = S.qlimit;
  ma.work_limit = S.work_limit;
  ma.seg_work = segwork;
  ma.abort_flag = d_err;
  ma.list = list_mode;
  ma.donate = donate;
  ma.timeout_cycles = (long long)timeout_ms * (long long)clock_khz;
  ma.split_min = split_min;
  ma.donate_depth = donate_depth;
  ma.pack_max = pack_max;
  ma.merge_max = merge_max;
  ma.out_seg = (uint32_t *)d_out_seg.ptr;
  ma.out_tup = (uint32_t *)d_out_tup.ptr;
  ma.cap = list_mode ? std::min<unsigned long long>(d_out_seg.bytes / 4, d_out_tup.bytes / 4 / ma.W) : 0;
  int blocks = num_sms * (warps_per_sm ? std::max(1, warps_per_sm / 8) : default_blocks_per_sm());

  const bool tuning = tune_next && S.match && !S.plain;
  const bool graphed = use_graph && !tuning && !S.plain;
  auto read_back = [&]() -> int {
    CK(cudaMemcpyAsync(h_sched.ptr, d_sched.ptr, sizeof(Sched), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync((char *)h_sched.ptr + sizeof(Sched), d_misc.ptr, 64, cudaMemcpyDeviceToHost, stream));
    if (S.nq_live)
      CK(cudaMemcpyAsync(h_qlisted.ptr, d_qlisted.ptr, (size_t)S.nq_live * 8, cudaMemcpyDeviceToHost, stream));
    return DSM_OK;
  };
  if (S.match && filter_mode > 0) filter_timed = true;  // a replayed graph records the filter events too
  if (graphed) {
    // everything the captured nodes bake in: pointers, settings, grids
    std::string key;
    key_append(key, ca);
    key_append(key, es);
    key_append(key, au);
    key_append(key, sa);
    key_append(key, ma);
    key_append(key, blocks);
    key_append(key, S.nq_live);
    key_append(key, S.match);
    key_append(key, query_gen);
    key_append(key, filter_mode);
    key_append(key, filter_incremental);
    key_append(key, bfs_levels);
    key_append(key, d_rows.ptr);
    key_append(key, d_rows.bytes);
    key_append(key, stall_test);
    key_append(key, h_sched.ptr);
    key_append(key, h_qlisted.ptr);
    rc = run_segment(0, key, [&]() -> int {
      if (int r = seg_a_kernels(S, ca, es, au, sa, true)) return r;
      if (S.match) {
        if (int r = rec(ev_pool[2])) return r;
        if (int r = launch_match_seq(ma, blocks, bfs_levels)) return r;
        if (int r = rec(ev_pool[3])) return r;
      }
      return read_back();
    });
    if (rc) return rc;
  } else {
    if ((rc = seg_a_kernels(S, ca, es, au, sa, !S.plain))) return rc;
    if (S.match) {
      if (tuning) {
        tune_next = false;
        if ((rc = autotune(ma, S, blocks))) return rc;
      }
      if ((rc = match_eager(S, ma, sa, blocks))) return rc;
    } else if ((rc = read_back())) {
      return rc;
    }
  }
  CK(cudaGetLastError());
  return DSM_OK;
}

// The matcher launch of a batch.  With breadth-first levels (label-major
// runs only) it is two launches: the first writes every prefix of 2 +
// `levels` positions to the row table instead of descending (while the
// table has room; beyond it, tasks go on depth-first), the second takes
// those rows as its tasks -- the reference's breadth-first expansion before
// its depth-first matcher (gpu_match.cu:1291-1357) and its row-by-row edge
// join (join.cu:106-221), in place of one launch per level.
int Engine::launch_match_seq(const MatchArgs &ma, int blocks, uint32_t levels) {
  if (levels == 0 || !ma.g.loff || !d_rows.ptr) {
    launch_match(ma, blocks, stream);
    ++stats.kernel_launches;
    return DSM_OK;
  }
  const unsigned long long cap = d_rows.bytes / sizeof(JobRec);
  unsigned long long *cnt = (unsigned long long *)((char *)d_misc.ptr + 160);
  CK(cudaMemsetAsync(cnt, 0, 8, stream));
  MatchArgs a1 = ma;
  a1.bfs_stop = 2 + levels;
  a1.rows_out = (JobRec *)d_rows.ptr;
  a1.rows_cnt = cnt;
  a1.rows_cap = cap;
  launch_match(a1, blocks, stream);
  launch_rows_arm((Sched *)d_sched.ptr, cnt, cap, stream);
  launch_sched_init((Sched *)d_sched.ptr, nullptr, (unsigned long long *)d_job_seq.ptr, job_ring, stream, stall_test);
  MatchArgs a2 = ma;
  a2.rows_in = (const JobRec *)d_rows.ptr;
  launch_match(a2, blocks, stream);
  stats.kernel_launches += 4;
  return DSM_OK;
}

// The matcher, eagerly: one launch for every query, or (plain form) one launch
// per query with a host round trip after each; the scheduler state of all of
// them is combined into h_sched.
int Engine::match_eager(Staged &S, MatchArgs &ma, SeedArgs &sa, int blocks) {
  const int sblocks = num_sms * 4;
  if (!S.plain) {
    if (int r = rec(ev_pool[2])) return r;
    if (int r = launch_match_seq(ma, blocks, bfs_levels)) return r;
    if (int r = rec(ev_pool[3])) return r;
    CK(cudaMemcpyAsync(h_sched.ptr, d_sched.ptr, sizeof(Sched), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync((char *)h_sched.ptr + sizeof(Sched), d_misc.ptr, 64, cudaMemcpyDeviceToHost, stream));
    if (S.nq_live)
      CK(cudaMemcpyAsync(h_qlisted.ptr, d_qlisted.ptr, (size_t)S.nq_live * 8, cudaMemcpyDeviceToHost, stream));
    return DSM_OK;
  }
  // plain: query by query, the result table filling on from where the last
  // query left it
  Sched total;
  std::memset(&total, 0, sizeof(total));
  Sched *hs = (Sched *)h_sched.ptr;
  unsigned long long out = 0;
  if (int r = rec(ev_pool[2])) return r;
  for (uint32_t ql = 0; ql < S.nq_live; ++ql) {
    std::memset(hs, 0, sizeof(Sched));
    hs->out_count.v = out;
    CK(cudaMemcpyAsync(d_sched.ptr, hs, sizeof(Sched), cudaMemcpyHostToDevice, stream));
    sa.only_slot = S.qids[ql];
    launch_seeds(sa, sblocks, stream);
    launch_sched_init((Sched *)d_sched.ptr, (const BatchHdr *)d_hdr.ptr, (unsigned long long *)d_job_seq.ptr,
                      job_ring, stream, stall_test);
    stats.kernel_launches += 2;
    if (int r = launch_match_seq(ma, blocks, bfs_levels)) return r;
    CK(cudaMemcpyAsync(hs, d_sched.ptr, sizeof(Sched), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    total.nseeds += hs->seeds ? hs->seeds : hs->nseeds;
    total.donations += hs->donations;
    total.steals += hs->steals;
    total.alg_bytes += hs->alg_bytes;
    total.matches += hs->matches;
    total.error |= hs->error;
    out = hs->out_count.v;
    if (hs->error) break;
  }
  total.out_count.v = out;
  if (int r = rec(ev_pool[3])) return r;
  std::memcpy(hs, &total, sizeof(Sched));
  CK(cudaMemcpyAsync((char *)h_sched.ptr + sizeof(Sched), d_misc.ptr, 64, cudaMemcpyDeviceToHost, stream));
  if (S.nq_live)
    CK(cudaMemcpyAsync(h_qlisted.ptr, d_qlisted.ptr, (size_t)S.nq_live * 8, cudaMemcpyDeviceToHost, stream));
  return DSM_OK;
}

int Engine::finish_device(Staged &S) {
  HostOut &H = hout[S.slot];
  CK(cudaStreamSynchronize(stream));
  const unsigned int *err0 = (const unsigned int *)((const char *)h_sched.ptr + sizeof(Sched));
  const bool arena_short = err0[0] & kErrArena;
  const uint64_t arena_need16 = ((const unsigned long long *)err0)[2];
  DevGraph g = dev_graph();
  const BatchHdr *dh = (const BatchHdr *)d_hdr.ptr;
  AdjUpdateArgs au{g, dh, (const unsigned long long *)d_dkey.ptr, (const uint32_t *)d_dhead.ptr,
                   (const unsigned long long *)d_bkey.ptr, (const uint8_t *)d_gflag.ptr, (uint32_t *)d_dsel.ptr,
                   (unsigned int *)d_misc.ptr, (unsigned long long *)((char *)d_misc.ptr + 8),
                   (unsigned long long *)((char *)d_misc.ptr + 16)};
  const int blocks = num_sms * 4;
  if (arena_short) {
    // nothing was written to the arena; the marks still go
    launch_clear_touch(g, dh, (const uint4 *)d_upd.ptr, blocks, stream);
    CK(cudaStreamSynchronize(stream));
    if (int rc = compact_arena(arena_need16 * 4)) return rc;
    return kRetryArena;
  }
  std::memcpy(&S.sc, h_sched.ptr, sizeof(Sched));
  S.qlisted.assign((const unsigned long long *)h_qlisted.ptr,
                   (const unsigned long long *)h_qlisted.ptr + S.nq_live);
  S.listed = list_mode && S.match;
  S.match_rc = DSM_OK;
  if (S.match) {
    MatchArgs ma;  // only for a rerun after the result table grew
    for (int attempt = 0;; ++attempt) {
      if (S.sc.error & kErrTimeout) {
        S.match_rc = fail(DSM_ERR_TIMEOUT, "matcher: a bounded wait gave up");
        break;
      }
      if (S.sc.error & kErrSeeds) {
        S.match_rc = fail(DSM_ERR_OVERFLOW, "seed table overflow");
        break;
      }
      if (!S.listed) break;
      // the counts are complete (the matcher counts past the capacity);
      // listing more than the batch limit downgrades the batch to counts
      const unsigned long long cap =
          std::min<unsigned long long>(d_out_seg.bytes / 4, d_out_tup.bytes / 4 / S.W);
      if ((double)S.sc.out_count.v * (S.W + 1) * 4.0 > (double)list_limit_bytes) {
        S.listed = 0;
        set_error("batch listing exceeds the listing limit; returned counts only");
        break;
      }
      if (S.sc.out_count.v <= cap) break;
      if (attempt >= 2) {
        S.match_rc = fail(DSM_ERR_OVERFLOW, "result table kept overflowing");
        break;
      }
      // grow to the exact count and run the matcher again on the same union graph
      // (a failure from here on still lets the batch's deletions run below:
      // the graph ends in the batch's final state and the batch reports it)
      ++stats.result_regrows;
      result_cap = S.sc.out_count.v + S.sc.out_count.v / 8 + 1024;
      if (int rc = dalloc(d_out_seg, result_cap * 4)) {
        S.match_rc = rc;
        break;
      }
      if (int rc = dalloc(d_out_tup, result_cap * S.W * 4)) {
        S.match_rc = rc;
        break;
      }
      Sched *hs = (Sched *)h_sched.ptr;
      const unsigned long long nseeds = S.sc.seeds ? S.sc.seeds : S.sc.nseeds;  // rows plan: nseeds counts rows
      std::memset(hs, 0, sizeof(Sched));
      hs->nseeds = nseeds;
      CK(cudaMemcpyAsync(d_sched.ptr, hs, sizeof(Sched), cudaMemcpyHostToDevice, stream));
      CK(cudaMemsetAsync(d_segcnt.ptr, 0, S.nseg * 8, stream));
      if (S.work_limit) CK(cudaMemsetAsync(d_segwork.ptr, 0, S.nseg * 8, stream));
      CK(cudaMemsetAsync(d_qlisted.ptr, 0, std::max<size_t>(S.nq_live, 1) * 8, stream));
      launch_sched_init((Sched *)d_sched.ptr, dh, (unsigned long long *)d_job_seq.ptr, job_ring, stream, stall_test);
      ++stats.kernel_launches;
      std::memset(&ma, 0, sizeof(ma));
      ma.g = g;
      ma.bt = DevBatchEdges{(const unsigned long long *)d_bkey.ptr, (const uint32_t *)d_binfo.ptr, 0};
      ma.hdr = dh;
      ma.vtp = (const uint32_t *)d_vtp.ptr;
      ma.qd = (const QDev *)d_qd.ptr;
      ma.orders = (const OrderRec *)d_orders.ptr;
      ma.seeds = (const uint4 *)d_seeds.ptr;
      ma.sc = (Sched *)d_sched.ptr;
      ma.jobs = (JobRec *)d_jobs.ptr;
      ma.job_seq = (unsigned long long *)d_job_seq.ptr;
      ma.job_ring = job_ring;
      ma.W = S.W;
      ma.seg_count = (unsigned long long *)d_segcnt.ptr;
      ma.qlisted = (unsigned long long *)d_qlisted.ptr;
      ma.qlimit = S.qlimit;
      ma.work_limit = S.work_limit;
      ma.seg_work = S.work_limit ? (unsigned long long *)d_segwork.ptr : nullptr;
      ma.abort_flag = (const unsigned int *)d_misc.ptr;
      ma.list = 1;
      ma.donate = donate;
      ma.timeout_cycles = (long long)timeout_ms * (long long)clock_khz;
      ma.split_min = split_min;
      ma.donate_depth = donate_depth;
      ma.pack_max = pack_max;
      ma.merge_max = merge_max;
      ma.out_seg = (uint32_t *)d_out_seg.ptr;
      ma.out_tup = (uint32_t *)d_out_tup.ptr;
      ma.cap = std::min<unsigned long long>(d_out_seg.bytes / 4, d_out_tup.bytes / 4 / S.W);
      const int mblocks = num_sms * (warps_per_sm ? std::max(1, warps_per_sm / 8) : default_blocks_per_sm());
      SeedArgs sa{g, dh, (const uint4 *)d_upd.ptr, (const uint32_t *)d_vtp.ptr, (const uint32_t *)d_pair_off.ptr,
                  (const uint32_t *)d_pair_ent.ptr, (const QDev *)d_qd.ptr, (const OrderRec *)d_orders.ptr,
                  (uint4 *)d_seeds.ptr, (Sched *)d_sched.ptr, kAllSlots};
      if (S.plain) {
        if (int rc = match_eager(S, ma, sa, mblocks)) {
          S.match_rc = rc;
          break;
        }
      } else {
        if (int r = rec(ev_pool[2])) return r;
        if (int r = launch_match_seq(ma, mblocks, bfs_levels)) return r;
        if (int r = rec(ev_pool[3])) return r;
        CK(cudaMemcpyAsync(h_sched.ptr, d_sched.ptr, sizeof(Sched), cudaMemcpyDeviceToHost, stream));
        if (S.nq_live)
          CK(cudaMemcpyAsync(h_qlisted.ptr, d_qlisted.ptr, (size_t)S.nq_live * 8, cudaMemcpyDeviceToHost,
                             stream));
      }
      CK(cudaStreamSynchronize(stream));
      std::memcpy(&S.sc, h_sched.ptr, sizeof(Sched));
      S.qlisted.assign((const unsigned long long *)h_qlisted.ptr,
                       (const unsigned long long *)h_qlisted.ptr + S.nq_live);
    }
    elapsed(ev_pool[2], ev_pool[3], &S.ms_match);
  }
  elapsed(H.ev0, ev_pool[1], &S.ms_upd);
  S.ms_filter = 0;
  if (filter_timed) {
    elapsed(ev_pool[5], ev_pool[6], &S.ms_filter);
    filter_timed = false;
  }

  // ---- segment B: deletions and marks; then the downloads
  S.cnt = (S.listed && S.match_rc == DSM_OK) ? (size_t)std::min<unsigned long long>(
                                                   S.sc.out_count.v, d_out_seg.bytes / 4)
                                             : 0;
  if (S.cnt) {
    if (int rc = halloc(H.out_seg, S.cnt * 4)) return rc;
    if (int rc = halloc(H.out_tup, S.cnt * S.W * 4)) return rc;
  }
  const bool graphed = use_graph && !S.plain;
  auto seg_b = [&]() -> int {
    launch_adj_delete(au, blocks, stream);
    launch_clear_touch(g, dh, (const uint4 *)d_upd.ptr, blocks, stream);
    stats.kernel_launches += 2;
    return DSM_OK;
  };
  if (graphed) {
    std::string key;
    key_append(key, au);
    key_append(key, blocks);
    if (int rc = run_segment(1, key, seg_b)) return rc;
  } else if (int rc = seg_b()) {
    return rc;
  }
  const size_t nn = std::max<uint32_t>(S.n, 1);
  if (S.cnt) {
    CK(cudaMemcpyAsync(H.out_seg.ptr, d_out_seg.ptr, S.cnt * 4, cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(H.out_tup.ptr, d_out_tup.ptr, S.cnt * S.W * 4, cudaMemcpyDeviceToHost, stream));
  }
  if (S.nq_live && S.n)
    CK(cudaMemcpyAsync(H.segcnt.ptr, d_segcnt.ptr, (size_t)S.nq_live * S.n * 8, cudaMemcpyDeviceToHost, stream));
  CK(cudaMemcpyAsync(H.vtp.ptr, d_vtp.ptr, nn * 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaMemcpyAsync(H.misc.ptr, d_misc.ptr, 64, cudaMemcpyDeviceToHost, stream));
  CK(cudaMemcpyAsync((char *)H.misc.ptr + 64, d_arena_top.ptr, 8, cudaMemcpyDeviceToHost, stream));
  CK(cudaEventRecord(H.ev_end, stream));
  CK(cudaGetLastError());
  // a long-running stream abandons the old runs of relocated lists: compact
  // (after this batch's device work, which the compaction waits for) once
  // the arena may be more than 7/8 used
  // (not fatal: this batch is complete; without room a later batch is
  // refused before it writes anything)
  const uint64_t top_bound = ((const unsigned long long *)err0)[3] + arena_need16;
  if (top_bound * 4 > arena_words - arena_words / 8 && compact_arena(0) != DSM_OK)
    set_error("arena compaction postponed: " + error_text());
  return DSM_OK;
}

int Engine::finish_or_retry(Staged &S) {
  int rc = finish_device(S);
  if (rc != kRetryArena) return rc;
  if ((rc = launch_front(S))) return rc;
  rc = finish_device(S);
  return rc == kRetryArena ? fail(DSM_ERR_OOM, "adjacency arena: no room for the batch even after compaction") : rc;
}

int Engine::run_front_and_finish(Staged &S) {
  if (int rc = launch_front(S)) return rc;
  return finish_or_retry(S);
}

int Engine::assemble(Staged &S, BatchResult &R) {
  HostOut &H = hout[S.slot];
  CK(cudaEventSynchronize(H.ev_end));
  const unsigned int *err = (const unsigned int *)H.misc.ptr;
  unsigned long long reloc = 0, top16 = 0;
  std::memcpy(&reloc, (const char *)H.misc.ptr + 8, 8);
  std::memcpy(&top16, (const char *)H.misc.ptr + 64, 8);
  if (err[0] & kErrArena) return fail(DSM_ERR_OOM, "adjacency arena full (relocation failed)");
  if (S.match_rc) return S.match_rc;
  float ms_total = 0;
  elapsed(H.ev0, H.ev_end, &ms_total);
  const uint32_t n = S.n, nql = S.nq_live;
  R.n = n;
  R.qids = S.qids;
  R.widths = S.widths;
  R.signs.assign(n, 0);
  const uint32_t *vtp = (const uint32_t *)H.vtp.ptr;
  for (uint32_t i = 0; i < n; ++i)
    if (vtp[i] != kNoView) R.signs[i] = S.ups[i].op ? 1 : -1;
  R.counts.assign((size_t)nql * n, 0);
  if (nql && n) std::memcpy(R.counts.data(), H.segcnt.ptr, (size_t)nql * n * 8);
  R.qlisted.assign(nql, S.listed ? 1 : 0);
  if (S.listed && S.qlimit)
    for (uint32_t ql = 0; ql < nql; ++ql)
      if (S.qlisted[ql] > S.qlimit) R.qlisted[ql] = 0;
  // a segment over the work limit (bit 63) lists nothing and its count is
  // partial; the batch's exact matches leave it out
  uint64_t exact = 0, incomplete = 0;
  for (uint64_t c : R.counts) {
    if (c & kCountIncomplete) ++incomplete;
    else exact += c;
  }
  R.offsets.assign((size_t)nql * n + 1, 0);
  for (uint32_t ql = 0; ql < nql; ++ql)
    for (uint32_t i = 0; i < n; ++i) {
      const size_t s = (size_t)ql * n + i;
      const bool lst = R.qlisted[ql] && !(R.counts[s] & kCountIncomplete);
      R.offsets[s + 1] = R.offsets[s] + (lst ? R.counts[s] * R.widths[ql] : 0);
    }
  R.listed = S.listed;
  R.tuples.clear();
  if (S.listed) {
    R.tuples.resize(R.offsets.back());
    const uint32_t *hs = (const uint32_t *)H.out_seg.ptr, *ht = (const uint32_t *)H.out_tup.ptr;
    const size_t nseg = (size_t)nql * n;
    if (S.cnt < (1u << 16)) {
      std::vector<uint64_t> cur(R.offsets.begin(), R.offsets.end() - 1);
      for (size_t r = 0; r < S.cnt; ++r) {
        const uint32_t s = hs[r];
        const uint32_t ql = s / n;
        if (!R.qlisted[ql] || (R.counts[s] & kCountIncomplete)) continue;  // partial tuples
        const uint32_t w = R.widths[ql];
        std::memcpy(&R.tuples[cur[s]], ht + r * S.W, w * 4);
        cur[s] += w;
      }
    } else {
      // on all host threads: each tuple claims its place in its segment by an
      // atomic cursor (the order inside a segment is the device's, which is
      // unordered anyway; the sort below makes it canonical)
      std::unique_ptr<std::atomic<uint64_t>[]> cur(new std::atomic<uint64_t>[nseg]);
      for (size_t k = 0; k < nseg; ++k) cur[k].store(R.offsets[k], std::memory_order_relaxed);
      parallel_for(S.cnt, 1u << 15, [&](size_t lo, size_t hi) {
        for (size_t r = lo; r < hi; ++r) {
          const uint32_t s = hs[r];
          const uint32_t ql = s / n;
          if (!R.qlisted[ql] || (R.counts[s] & kCountIncomplete)) continue;  // partial tuples
          const uint32_t w = R.widths[ql];
          const uint64_t p = cur[s].fetch_add(w, std::memory_order_relaxed);
          std::memcpy(&R.tuples[p], ht + r * S.W, w * 4);
        }
      });
    }
    if (S.sort) {
      std::vector<uint64_t> cnt_listed(R.counts);
      for (uint32_t ql = 0; ql < nql; ++ql)
        for (uint32_t i = 0; i < n; ++i) {
          uint64_t &c = cnt_listed[(size_t)ql * n + i];
          if (!R.qlisted[ql] || (c & kCountIncomplete)) c = 0;
        }
      const auto ts = std::chrono::steady_clock::now();
      sort_segments(R, cnt_listed, nql, n, S.cnt);
      R.sort_ms = ms_since(ts);
    }
  }
  R.device_ms = ms_total;
  R.match_ms = S.ms_match;
  R.host_prep_ms = S.host_prep_ms;
  R.alg_bytes = S.sc.alg_bytes;
  R.matches = exact;
  R.incomplete = incomplete;
  {
    std::lock_guard<std::mutex> lk(smu);
    stats.batches++;
    stats.updates += n;
    stats.matches += exact;
    stats.over_limit += incomplete;
    stats.seeds += S.sc.seeds ? S.sc.seeds : S.sc.nseeds;
    stats.donations += S.sc.donations;
    stats.steals += S.sc.steals;
    stats.relocations += reloc;
    stats.alg_bytes += S.sc.alg_bytes;
    stats.last_batch_ms = ms_total;
    stats.last_match_ms = S.ms_match;
    stats.last_update_ms = S.ms_upd;
    stats.last_filter_ms = S.ms_filter;
    stats.last_sort_ms = R.sort_ms;
  }
  (void)top16;
  return DSM_OK;
}

int Engine::run_batch(const dsm_update *ups, uint32_t n, BatchResult &R, bool match) {
  Staged S;
  const int slot = next_slot;
  next_slot ^= 1;
  if (int rc = prepare(ups, n, S, slot)) return rc;
  S.match = match;
  if (int rc = run_front_and_finish(S)) return rc;
  return assemble(S, R);
}

// ---------------------------------------------------------------------------
// arena compaction
// ---------------------------------------------------------------------------
// Every run moves to a fresh arena in vertex order with the load-time slack
// (capacity = deg + deg / 8 + 4, rounded to 4), and the arena keeps a quarter
// plus `extra_words` free.  Slot offsets index within runs and stay valid.
int Engine::compact_arena(uint64_t extra_words) {
  CK(cudaStreamSynchronize(stream));
  std::vector<uint2> adj(nv), nadj(nv);
  std::vector<uint32_t> ncap(nv);
  CK(cudaMemcpy(adj.data(), d_adj.ptr, (size_t)nv * 8, cudaMemcpyDeviceToHost));
  uint64_t off16 = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    const uint32_t d = adj[v].y;
    ncap[v] = (d + d / 8 + 4 + 3) & ~3u;
    nadj[v] = make_uint2((uint32_t)off16, d);
    off16 += ncap[v] / 4;
  }
  if (off16 > 0xFFFFFFFFull) return fail(DSM_ERR_LIMIT, "graph too large for 32-bit run offsets");
  uint64_t words = off16 * 4 + off16 + extra_words + std::min<uint64_t>(off16 * 4, 1u << 20);
  words = (words + 3) & ~3ull;
  DevBuf na, nadj_d, ncap_d;
  int rc;
  if ((rc = dalloc(na, words * 4)) || (rc = dalloc(nadj_d, (size_t)nv * 8)) || (rc = dalloc(ncap_d, (size_t)nv * 4))) {
    dfree(na);
    dfree(nadj_d);
    dfree(ncap_d);
    return rc;
  }
  CK(cudaMemcpyAsync(nadj_d.ptr, nadj.data(), (size_t)nv * 8, cudaMemcpyHostToDevice, stream));
  launch_arena_move(dev_graph(), (const uint2 *)nadj_d.ptr, (uint32_t *)na.ptr, num_sms * 8, stream);
  CK(cudaMemcpyAsync(d_adj.ptr, nadj_d.ptr, (size_t)nv * 8, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(d_cap.ptr, ncap.data(), (size_t)nv * 4, cudaMemcpyHostToDevice, stream));
  unsigned long long top = off16;
  CK(cudaMemcpyAsync(d_arena_top.ptr, &top, 8, cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  CK(cudaGetLastError());
  dfree(d_arena);
  d_arena = na;
  dfree(nadj_d);
  dfree(ncap_d);
  arena_words = words;
  arena_used16 = off16;
  ++compactions;
  stats.compactions = compactions;
  ++query_gen;  // captured graphs hold the old arena
  return DSM_OK;
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
// The matcher's result does not depend on its launch shape or on how work is
// donated, so the batch's own matcher launch is repeated on the same union
// graph (counts only) for each candidate -- first the intersection tile
// (packed last level), then resident blocks per SM x range-split threshold x
// donation depth at the best tile -- timed with events, and the fastest
// becomes the engine's setting.  The first candidate runs twice and its first
// run is not counted (it warms L2 for all).
int Engine::autotune(MatchArgs &ma, const Staged &S, int &blocks) {
  Sched *hs = (Sched *)h_sched.ptr;
  CK(cudaMemcpyAsync(hs, d_sched.ptr, sizeof(Sched), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (hs->error) return DSM_OK;  // the real launch reports it
  const unsigned long long nseeds = hs->nseeds;
  struct Cand {
    int bps;
    uint32_t split, dd, pack, merge, bfs;
  };
  auto rearm = [&]() -> int {
    std::memset(hs, 0, sizeof(Sched));
    hs->nseeds = nseeds;
    CK(cudaMemcpyAsync(d_sched.ptr, hs, sizeof(Sched), cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(d_segcnt.ptr, 0, S.nseg * 8, stream));
    if (S.work_limit) CK(cudaMemsetAsync(d_segwork.ptr, 0, S.nseg * 8, stream));
    CK(cudaMemsetAsync(d_qlisted.ptr, 0, std::max<size_t>(S.nq_live, 1) * 8, stream));
    launch_sched_init((Sched *)d_sched.ptr, (const BatchHdr *)d_hdr.ptr, (unsigned long long *)d_job_seq.ptr,
                      job_ring, stream, stall_test);
    ++stats.kernel_launches;
    CK(cudaStreamSynchronize(stream));  // hs is read by the copy
    return DSM_OK;
  };
  MatchArgs t = ma;
  t.list = 0;
  t.cap = 0;
  cudaEvent_t e0 = ev_pool[2], e1 = ev_pool[3];
  // times each candidate; bc = the fastest (unchanged when a launch reports
  // an error in the scheduler word: the batch's real launch reports it)
  bool stop = false;
  auto sweep = [&](const std::vector<Cand> &cands, bool warm, Cand &bc, float &best) -> int {
    best = 1e30f;
    for (int k = warm ? -1 : 0; k < (int)cands.size() && !stop; ++k) {
      const Cand &c = cands[std::max(k, 0)];
      if (int rc = rearm()) return rc;
      t.split_min = c.split;
      t.donate_depth = c.dd;
      t.pack_max = c.pack;
      t.merge_max = c.merge;
      CK(cudaEventRecord(e0, stream));
      if (int r = launch_match_seq(t, num_sms * c.bps, c.bfs)) return r;
      CK(cudaEventRecord(e1, stream));
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(hs, d_sched.ptr, sizeof(Sched), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      if (hs->error) {
        stop = true;
        break;
      }
      float ms = 0;
      elapsed(e0, e1, &ms);
      stats.tune_runs++;
      if (k >= 0 && ms < best) {
        best = ms;
        bc = c;
      }
    }
    return DSM_OK;
  };
  const Cand cur{blocks / std::max(num_sms, 1), ma.split_min, ma.donate_depth, ma.pack_max, ma.merge_max,
                 bfs_levels};
  // stage 0: depth-first or breadth-first rows for the first 1 or 2 levels
  std::vector<Cand> c0;
  for (uint32_t bl : {0u, 1u, 2u}) c0.push_back({cur.bps, cur.split, cur.dd, cur.pack, cur.merge, bl});
  float best0 = 1e30f, best1 = 1e30f, best2 = 1e30f;
  Cand b0 = cur;
  if (d_rows.ptr)
    if (int rc = sweep(c0, true, b0, best0)) return rc;
  // stage 1: the intersection tile -- packed last level x merge threshold --
  // at the current launch shape
  std::vector<Cand> c1;
  for (uint32_t pk : {0u, 256u, 1024u, 4096u})
    for (uint32_t mg : {0u, 64u, 256u}) c1.push_back({cur.bps, cur.split, cur.dd, pk, mg, b0.bfs});
  Cand b1 = b0, bc = b0;
  if (!stop)
    if (int rc = sweep(c1, !d_rows.ptr, b1, best1)) return rc;
  // stage 2: blocks per SM x split threshold x donation depth, at that tile
  std::vector<Cand> c2;
  for (int bps = std::max(1, match_blocks_per_sm - 2); bps <= match_blocks_per_sm; ++bps)
    for (uint32_t split : {64u, 128u, 512u})
      for (uint32_t dd : {1u, 2u}) c2.push_back({bps, split, dd, b1.pack, b1.merge, b1.bfs});
  bc = b1;
  if (!stop)
    if (int rc = sweep(c2, false, bc, best2)) return rc;
  if (!stop && best2 < 1e30f) {
    warps_per_sm = bc.bps * 8;
    split_min = bc.split;
    donate_depth = bc.dd;
    pack_max = bc.pack;
    merge_max = bc.merge;
    bfs_levels = bc.bfs;
    stats.tune_best_ms = best2;
  }
  ma.pack_max = pack_max;
  ma.merge_max = merge_max;
  ma.split_min = split_min;
  ma.donate_depth = donate_depth;
  blocks = num_sms * (warps_per_sm ? std::max(1, warps_per_sm / 8) : default_blocks_per_sm());
  return rearm();  // the batch's real launch starts from scratch
}

// ---------------------------------------------------------------------------
// CUDA-graph replay
// ---------------------------------------------------------------------------
// Segment k is captured once and replayed while `key` -- every pointer,
// setting and grid its nodes bake in -- stays the same; the kernels read the
// batch's sizes from the device header, so batches of any size replay it.
// A new key re-captures: the executable graph is updated in place when the
// topology is unchanged, else instantiated anew.
int Engine::run_segment(int k, const std::string &key, const std::function<int()> &fn) {
  if (gexec[k] && gkey[k] == key) {
    CK(cudaGraphLaunch(gexec[k], stream));
    stats.graph_launches++;
    stats.kernel_launches += seg_kernels[k];  // the kernels the replayed graph holds
    return DSM_OK;
  }
  CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  capturing = true;
  const uint64_t launches0 = stats.kernel_launches;
  const int rc = fn();
  seg_kernels[k] = stats.kernel_launches - launches0;
  capturing = false;
  cudaGraph_t gr = nullptr;
  const cudaError_t e = cudaStreamEndCapture(stream, &gr);
  if (rc || e != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    cudaGetLastError();
    gkey[k].clear();
    return rc ? rc : cuda_fail(e, "graph capture");
  }
  stats.graph_captures++;
  bool updated = false;
  if (gexec[k]) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(gexec[k], gr, &info) == cudaSuccess) {
      updated = true;
    } else {
      cudaGetLastError();
      cudaGraphExecDestroy(gexec[k]);
      gexec[k] = nullptr;
    }
  }
  if (!updated) {
    const cudaError_t ei = cudaGraphInstantiate(&gexec[k], gr, 0);
    if (ei != cudaSuccess) {
      cudaGraphDestroy(gr);
      gexec[k] = nullptr;
      gkey[k].clear();
      return cuda_fail(ei, "graph instantiate");
    }
    stats.graph_instantiations++;
  }
  cudaGraphDestroy(gr);
  gkey[k] = key;
  CK(cudaGraphLaunch(gexec[k], stream));
  stats.graph_launches++;
  return DSM_OK;
}

}  // namespace dsm
