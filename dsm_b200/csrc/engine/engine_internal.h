// Engine object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/dsm.h"
#include "../host/query_plan.h"
#include "common.cuh"
#include "filter.cuh"
#include "kernels.cuh"

namespace dsm {

const char *status_string(int s);

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
};
struct HostBuf {
  void *ptr = nullptr;  // pinned
  size_t bytes = 0;
};

struct Slot {
  bool live = false;
  QueryPlan plan;
  DevBuf bitmap;          // nq x col_len candidate bitmaps
  DevBuf filter_scratch;  // vcand, valid, encodings (per data vertex)
  DevBuf filter_plan;     // QFilterDesc + op list
  uint32_t filter_nops = 0;
  uint32_t filter_hops = 0;  // hops of its incremental region (> kRegionMaxHops: always full)
  bool filter_dirty = true;  // plan or sizes must be (re)uploaded
  size_t foot = 0;           // device bytes charged to this query at admission
};

// Pinned host side of one device batch in flight (two sets, so the serving
// loop can assemble batch k on the host while batch k + 1 runs).
struct HostOut {
  HostBuf stage;   // uploads: updates, sorted keys, indices, directed pairs, group heads
  HostBuf hdr;     // BatchHdr
  HostBuf segcnt, vtp, out_seg, out_tup, misc;
  cudaEvent_t ev0 = nullptr, ev_end = nullptr;  // batch start, results downloaded
};

// One device batch from host preparation to result assembly.
struct Staged {
  const dsm_update *ups = nullptr;  // the caller's updates, valid until assemble
  uint32_t n = 0, m = 0, ngroups = 0;
  size_t ndir = 0;
  size_t o_up = 0, o_bk = 0, o_bi = 0, o_dk = 0, o_dh = 0;  // offsets in the staging buffer
  int slot = 0;
  bool match = true;  // false: apply the updates to the graph only
  double host_prep_ms = 0;
  // fixed at launch
  std::vector<uint32_t> qids, widths;
  uint32_t nq_live = 0, W = 1;
  size_t nseg = 0;
  unsigned long long seed_cap = 0;
  int plain = 0, sort = 1;
  unsigned long long qlimit = 0, work_limit = 0;
  // after the matcher
  Sched sc{};
  std::vector<unsigned long long> qlisted;
  int listed = 0, match_rc = 0;
  size_t cnt = 0;  // listed tuples downloaded
  float ms_match = 0, ms_upd = 0, ms_filter = 0;
};

struct BatchResult {
  uint64_t id = 0;
  uint32_t n = 0;
  std::vector<uint32_t> qids, widths;
  std::vector<uint8_t> qlisted;  // per query: its tuples are listed
  std::vector<int8_t> signs;
  std::vector<uint64_t> counts, offsets;
  std::vector<uint32_t> tuples;
  int listed = 1;
  double device_ms = 0, match_ms = 0, host_prep_ms = 0, sort_ms = 0;
  uint64_t alg_bytes = 0, matches = 0, incomplete = 0;
  // served timing: submit -> start of the device batch -> results readable
  double queue_ms = 0, service_ms = 0, total_ms = 0;
  uint32_t merged_requests = 1, merged_updates = 0;
};

// A request of the serving loop, in submission order.
enum ReqKind { kReqBatch = 0, kReqRegister = 1, kReqRetire = 2 };
struct Request {
  int kind = kReqBatch;
  uint64_t id = 0;  // batch id, or the ticket of a registration / retirement
  std::vector<dsm_update> ups;
  QueryPlan plan;   // registration (planned and validated at submit)
  uint32_t qid = 0; // retirement
  std::chrono::steady_clock::time_point t_submit;
};
struct Outcome {
  int rc = DSM_OK;
  uint32_t qid = 0;
  std::string msg;
};

// Serving loop: one worker thread drains the request queue.  Consecutive
// batches are merged into one device batch of at most max_merge updates;
// registrations and retirements take effect between device batches, in
// submission order.  A registration whose footprint does not fit now waits
// (FIFO) until retirements free memory.
struct Server {
  bool running = false, stopping = false;
  std::thread worker;
  std::mutex qmu;  // queue, pending, tickets, done, failed
  std::condition_variable work_cv, done_cv;
  std::deque<Request> queue;
  std::deque<Request> pending;
  // Bookkeeping stays bounded by what is in flight or unreported: a ticket
  // sits in open_tickets until its outcome is posted to `tickets`, and leaves
  // `tickets` once dsm_query_admission reported it; a queued batch sits in
  // `inflight` until its results (or failure) are final, and a failure leaves
  // `failed` once a wait reported it.
  std::set<uint64_t> open_tickets;
  std::map<uint64_t, Outcome> tickets;
  std::set<uint64_t> inflight;
  std::map<uint64_t, Outcome> failed;
  uint32_t max_merge = 65536;
  uint64_t next_ticket = 1;
};

struct Engine {
  int device = 0;
  size_t budget = 0;
  size_t bytes_in_use = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  int clock_khz = 1965000;
  int match_blocks_per_sm = 2;  // most resident matcher blocks per SM (the tuner's upper end)
  // untuned launch shape: 4 blocks per SM, the 64-register variant (the
  // 48-register one spills; tuning on config 2 and 4 picked 4 and 3 blocks)
  int default_blocks_per_sm() const { return std::max(1, std::min(match_blocks_per_sm, 4)); }
  std::mutex mu;
  std::mutex emu;          // guards last_error (written by the serving worker too)
  std::string last_error;
  void set_error(const std::string &m) {
    std::lock_guard<std::mutex> lk(emu);
    last_error = m;
  }
  std::string error_text() {
    std::lock_guard<std::mutex> lk(emu);
    return last_error;
  }
  std::vector<cudaEvent_t> ev_pool;

  // options
  int list_mode = 1;
  int filter_mode = 0;
  int donate = 1;
  int warps_per_sm = 0;
  int64_t timeout_ms = 5000;
  int label_quirk = 0;
  int sort_results = 1;
  uint32_t split_min = 0, donate_depth = 0;  // donation granularity (0 = kernel default)
  uint32_t pack_max = 1024;                  // packed last level (entries per pass; 0: off)
  uint32_t merge_max = 64;                   // merge intersection up to this probe range (0: off)
  uint32_t bfs_levels = 0;                   // breadth-first rows: levels beyond the seed (0: depth-first)
  uint64_t bfs_rows = 1u << 20;              // row table capacity
  DevBuf d_rows;
  bool tune_next = false;                    // autotune on the next batch
  int use_graph = 0;                         // replay the batch segments as CUDA graphs
  int stall_test = 0;                        // arm matcher launches with a task nobody finishes
  int plain = 0;                             // one matcher launch per query (the reference's form)
  unsigned long long query_list_limit = 0;   // tuples one query may list per batch (0: no budget)
  unsigned long long work_limit = 0;         // partial embeddings per (query, update) (0: no limit)
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  std::string gkey[2];                       // what each executable graph was captured with
  uint64_t seg_kernels[2] = {0, 0};          // kernels each executable graph holds
  uint64_t query_gen = 0;                    // bumped whenever the live queries or filters change
  bool filter_timed = false;  // the filter events of this batch were recorded
  uint64_t result_cap = 1 << 20;
  uint32_t job_ring = 1 << 19;  // job slots of the matcher's donation ring
  uint64_t list_limit_bytes = 8ull << 30;  // beyond this a batch returns counts only

  // graph
  bool graph_loaded = false;
  uint32_t nv = 0;
  uint64_t arena_words = 0, arena_used16 = 0, graph_entries = 0;
  uint32_t nlt = 0;  // label slots in use (slot offsets per vertex: nlt + 1)
  std::vector<uint32_t> label_host;
  DevBuf d_lab, d_adj, d_cap, d_arena, d_arena_top, d_loff;
  // incremental filter region (filter.cuh RegionInfo)
  DevBuf d_rinfo, d_rmark, d_rlist, d_rprev;
  uint64_t region_batches = 0;  // filtered batches since the region buffers were set up
  int filter_incremental = 1;

  // queries
  std::vector<Slot> slots;
  bool queries_dirty = true, qd_dirty = true;
  std::vector<uint32_t> live_ids;
  std::vector<QDev> qd_host;
  uint32_t max_width = 0, max_bucket = 0;
  DevBuf d_qd, d_orders, d_pair_off, d_pair_ent;

  // batch scratch
  DevBuf d_upd, d_bkey, d_bidx, d_binfo, d_gflag, d_vtp, d_dkey, d_dhead, d_dsel, d_seeds, d_sched, d_jobs,
      d_job_seq, d_out_seg, d_out_tup, d_segcnt, d_misc, d_hdr, d_qlisted, d_segwork;
  HostBuf h_sched;    // Sched + the error words, read after the matcher
  HostBuf h_qlisted;  // per-query listing counters, read after the matcher
  HostOut hout[2];
  int next_slot = 0;
  uint64_t compactions = 0;

  // results (own lock: a waiter reads batch k while batch k + 1 runs)
  std::mutex rmu;
  std::map<uint64_t, std::unique_ptr<BatchResult>> results;
  std::atomic<uint64_t> next_batch_id{1};
  dsm_stats stats{};
  Server srv;

  ~Engine();
  int init(int device, size_t budget);
  int fail(int code, const std::string &msg);
  int cuda_fail(cudaError_t e, const char *where);
  int dalloc(DevBuf &b, size_t bytes);
  void dfree(DevBuf &b);
  int halloc(HostBuf &b, size_t bytes);
  std::vector<DevBuf *> all_dev_bufs();

  int load_graph(uint32_t nv, const uint32_t *labels, std::vector<uint64_t> &keys);
  uint32_t entry_of(uint32_t v) const { return pack_entry(label_host[v], v); }
  DevGraph dev_graph();
  int export_graph(uint32_t *offsets, uint32_t *nbrs, uint64_t *num_entries);
  int export_graph_locked(uint32_t *offsets, uint32_t *nbrs, uint64_t *num_entries);
  int snapshot(const char *path);  // snapshot.cu
  int resume(const char *path);

  int register_query(const uint32_t *qoff, const uint32_t *qnbr, const uint32_t *qlab, uint32_t nq, uint32_t *qid);
  int retire_query(uint32_t qid);
  size_t query_footprint(const QueryPlan &p) const;
  size_t query_bytes_allocated() const;
  int admit(QueryPlan &plan, uint32_t *qid, bool *fits_later, int64_t want_id = -1);  // mu held
  int retire_locked(uint32_t qid);                              // mu held
  int sync_queries();
  int upload_qd();
  int prepare_filters();
  int launch_filters();
  int run_segment(int k, const std::string &key, const std::function<int()> &fn);
  int rec(cudaEvent_t ev);
  void elapsed(cudaEvent_t a, cudaEvent_t b, float *ms);
  bool capturing = false;
  int prepare_filter(uint32_t id);
  int launch_filter(uint32_t id, int mode, int force_full);
  int launch_match_seq(const MatchArgs &ma, int blocks, uint32_t levels);
  RegionDevice region_dev();
  int region_init();
  int filter_state(uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us, uint32_t *info);
  int query_filter(uint32_t qid, uint32_t *bitmaps, uint32_t *v_cand_us);

  int check_updates(const dsm_update *ups, uint32_t n);
  int autotune(MatchArgs &ma, const Staged &S, int &blocks);
  int submit(const dsm_update *ups, uint32_t n, uint64_t *batch_id);
  int graph_apply(const dsm_update *ups, uint32_t n);
  // The batch pipeline (batch.cu): prepare (host only: sorted keys into the
  // slot's pinned staging), launch_front (mu held: uploads, edge state, union
  // insert, filters, seeds, matcher), finish_device (mu held: waits for the
  // matcher, regrows and reruns on overflow, enqueues deletions and the
  // downloads), assemble (host: waits for the downloads, builds the result).
  // run_batch chains them; the serving loop overlaps assemble of batch k
  // with the device work of batch k + 1.
  int prepare(const dsm_update *ups, uint32_t n, Staged &S, int slot);
  int launch_front(Staged &S);
  int finish_device(Staged &S);
  int assemble(Staged &S, BatchResult &R);
  int run_batch(const dsm_update *ups, uint32_t n, BatchResult &R, bool match = true);
  int run_front_and_finish(Staged &S);  // launch_front + finish_or_retry
  int finish_or_retry(Staged &S);       // finish_device; on a refused batch, compact and run it again
  int compact_arena(uint64_t extra_words);
  int match_eager(Staged &S, MatchArgs &ma, SeedArgs &sa, int blocks);  // one launch, or one per query
  int seg_a_kernels(Staged &S, const ClearArgs &ca, const EdgeStateArgs &es, const AdjUpdateArgs &au,
                    const SeedArgs &sa, bool seeds);
  std::mutex smu;  // stats written by assemble
  int wait_batch(uint64_t id);
  void sort_segments(BatchResult &R, const std::vector<uint64_t> &counts, uint32_t nq_live, uint32_t n,
                     size_t total);
  int view(uint64_t id, dsm_result_view *v);
  int release(uint64_t id);
  int timing(uint64_t id, dsm_batch_timing *t);

  // serving loop (serve.cu)
  int serve_start(uint32_t max_merge);
  int serve_stop();
  int register_async(const uint32_t *qoff, const uint32_t *qnbr, const uint32_t *qlab, uint32_t nq,
                     uint64_t *ticket);
  int retire_async(uint32_t qid, uint64_t *ticket);
  int admission(uint64_t ticket, int64_t timeout_ms, uint32_t *qid);
  void worker_loop();
  Outcome handle_control(Request &r);
  void post_batch(struct InFlight &b);
  void fail_batch(struct InFlight &b, int rc);
  void admit_pending();
  void post_outcome(uint64_t ticket, const Outcome &o);  // qmu held
};

}  // namespace dsm
