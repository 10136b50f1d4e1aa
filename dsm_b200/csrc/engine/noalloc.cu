// dsm_count_edge_embeddings_noalloc: the persistent matcher, counting only,
// with every piece of scratch it needs in one fixed device array.
//
// Some callers cannot allocate device memory while they run: code inside a
// host framework that owns the device allocator and forbids side allocations
// (a serving runtime with a pre-sized memory pool, an inference server that
// budgets every byte up front), or a thread that must not call cudaMalloc /
// cudaFree because those calls synchronise the whole device.  This entry
// point serves them: the caller passes its own device graph, updates and
// output, and the matcher's scheduler state, donation ring, seed table and
// query descriptor live in `g_na_scratch`, a file-scope array that every GPU
// loading this library holds (about 12.5 MB) until the process exits.
//
// Calls share that array and it keeps the last call's contents; each call
// clears what must start at zero.  Two calls whose work overlaps on the GPU
// (other streams, other threads) race on it and give wrong counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../../include/dsm.h"
#include "../host/query_plan.h"
#include "kernels.cuh"

namespace dsm {

namespace {

constexpr uint32_t kNaMaxUpdates = 4096;     // updates per call
constexpr uint32_t kNaMaxQueryVertices = 8;  // so at most 2 x 28 ordered query edges
constexpr uint32_t kNaMaxOrders = 56;
constexpr uint32_t kNaRing = 1u << 16;       // donation ring slots
constexpr size_t kNaSeedCap = (size_t)kNaMaxUpdates * kNaMaxOrders;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffSched = 0;
constexpr size_t kOffSeq = align256(kOffSched + sizeof(Sched));
constexpr size_t kOffJobs = align256(kOffSeq + 8ull * kNaRing);
constexpr size_t kOffSeeds = align256(kOffJobs + sizeof(JobRec) * (size_t)kNaRing);
constexpr size_t kOffQd = align256(kOffSeeds + 16 * kNaSeedCap);
constexpr size_t kOffOrders = align256(kOffQd + sizeof(QDev));
constexpr size_t kOffPairOff = align256(kOffOrders + sizeof(OrderRec) * kNaMaxOrders);
constexpr size_t kOffPairEnt = align256(kOffPairOff + 4 * (32 * 32 + 1));
constexpr size_t kOffVtp = align256(kOffPairEnt + 4 * kNaMaxOrders);
constexpr size_t kOffHdr = align256(kOffVtp + 4 * (size_t)kNaMaxUpdates);  // BatchHdr, then a zero word
constexpr size_t kScratchBytes = align256(kOffHdr + sizeof(BatchHdr) + 16);

static __device__ __align__(256) unsigned char g_na_scratch[kScratchBytes];

// Device address of g_na_scratch per device.  In host code the array's name
// is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
std::mutex g_na_mu;
unsigned char *g_na_addr[256] = {};

int scratch_of(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (device < 0 || device >= 256) return DSM_ERR_ARG;
  if (!g_na_addr[device]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return DSM_ERR_CUDA;
    }
    g_na_addr[device] = (unsigned char *)p;
  }
  *out = g_na_addr[device];
  return DSM_OK;
}

}  // namespace
}  // namespace dsm

extern "C" int dsm_count_edge_embeddings_noalloc(int device, uint32_t nv, const uint32_t *d_adj,
                                                 const uint32_t *d_arena, const uint32_t *d_labels,
                                                 const uint32_t *q_offsets, const uint32_t *q_nbrs,
                                                 const uint32_t *q_labels, uint32_t nq,
                                                 const dsm_update *d_updates, uint32_t n,
                                                 uint64_t *d_counts, void *stream) {
  using namespace dsm;
  if (!d_adj || !d_arena || !d_labels || !q_offsets || !q_nbrs || !q_labels || !d_counts || (n && !d_updates))
    return DSM_ERR_ARG;
  if (n > kNaMaxUpdates || nq > kNaMaxQueryVertices) return DSM_ERR_LIMIT;
  QueryPlan plan;
  std::string err;
  int rc = plan_query(nq, q_offsets, q_nbrs, q_labels, plan, err);
  if (rc) return rc;
  if (plan.orders.size() > kNaMaxOrders) return DSM_ERR_LIMIT;

  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return DSM_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return DSM_ERR_ARG;
  }
  auto done = [&](int code) {
    cudaSetDevice(prev);
    return code;
  };
  cudaStream_t s = (cudaStream_t)stream;
  // after the first asynchronous call, a failure waits for the work already
  // queued on the stream: it may still write the shared scratch and the
  // caller's counts, and a retry must not overlap it
  auto cuda_failed = [&]() {
    cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaGetLastError();
    return done(DSM_ERR_CUDA);
  };
  unsigned char *base = nullptr;
  if ((rc = scratch_of(device, &base))) return done(rc);

  // query descriptor, orders and the (label, label) -> ordered edge table
  QDev qd;
  std::memset(&qd, 0, sizeof(qd));
  qd.nq = nq;
  qd.n_orders = (uint32_t)plan.orders.size();
  for (uint32_t u = 0; u < nq; ++u) qd.label[u] = plan.labels[u];
  qd.col_len = (nv + 31) / 32;
  std::vector<uint32_t> pair_off(32 * 32 + 1, 0), pair_ent;
  {
    std::vector<std::vector<uint32_t>> buckets(32 * 32);
    for (size_t o = 0; o < plan.orders.size(); ++o)
      buckets[plan.labels[plan.oedges[o].first] * 32 + plan.labels[plan.oedges[o].second]].push_back((uint32_t)o);
    for (size_t b = 0; b < buckets.size(); ++b) {
      pair_off[b + 1] = pair_off[b] + (uint32_t)buckets[b].size();
      pair_ent.insert(pair_ent.end(), buckets[b].begin(), buckets[b].end());
    }
  }
  Sched *sc = (Sched *)(base + kOffSched);
  unsigned long long *seq = (unsigned long long *)(base + kOffSeq);
  uint32_t *vtp = (uint32_t *)(base + kOffVtp);
  BatchHdr hdr;
  std::memset(&hdr, 0, sizeof(hdr));
  hdr.n = n;
  hdr.nq_live = 1;
  hdr.seed_cap = kNaSeedCap;
  hdr.nseg = n;
  bool ok = cudaMemsetAsync(sc, 0, sizeof(Sched), s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffHdr, &hdr, sizeof(hdr), cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemsetAsync(base + kOffHdr + sizeof(BatchHdr), 0, 16, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffQd, &qd, sizeof(qd), cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffOrders, plan.orders.data(), plan.orders.size() * sizeof(OrderRec),
                            cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(base + kOffPairOff, pair_off.data(), pair_off.size() * 4, cudaMemcpyHostToDevice, s) ==
                cudaSuccess &&
            (pair_ent.empty() || cudaMemcpyAsync(base + kOffPairEnt, pair_ent.data(), pair_ent.size() * 4,
                                                 cudaMemcpyHostToDevice, s) == cudaSuccess) &&
            (n == 0 || cudaMemsetAsync(vtp, 0, 4ull * n, s) == cudaSuccess) &&
            (n == 0 || cudaMemsetAsync(d_counts, 0, 8ull * n, s) == cudaSuccess);
  if (!ok) return cuda_failed();

  // the caller's graph: adj = {run start in 16-byte units, degree} per vertex
  DevGraph g;
  std::memset(&g, 0, sizeof(g));
  g.nv = nv;
  g.lab = const_cast<uint32_t *>(d_labels);
  g.adj = reinterpret_cast<uint2 *>(const_cast<uint32_t *>(d_adj));
  g.arena = const_cast<uint32_t *>(d_arena);

  const BatchHdr *dh = (const BatchHdr *)(base + kOffHdr);
  SeedArgs sa{g, dh, reinterpret_cast<const uint4 *>(d_updates), vtp, (const uint32_t *)(base + kOffPairOff),
              (const uint32_t *)(base + kOffPairEnt), (const QDev *)(base + kOffQd),
              (const OrderRec *)(base + kOffOrders), (uint4 *)(base + kOffSeeds), sc, kAllSlots};
  int sms = 0, clk_khz = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device);
  launch_seeds(sa, std::max(sms, 1) * 4, s);
  launch_sched_init(sc, dh, seq, kNaRing, s);

  MatchArgs ma;
  std::memset(&ma, 0, sizeof(ma));
  ma.g = g;
  ma.bt = DevBatchEdges{nullptr, nullptr, 0};  // a fixed graph: every edge is live
  ma.vtp = vtp;
  ma.hdr = dh;
  ma.abort_flag = (const unsigned int *)(base + kOffHdr + sizeof(BatchHdr));
  ma.qd = (const QDev *)(base + kOffQd);
  ma.orders = (const OrderRec *)(base + kOffOrders);
  ma.seeds = (const uint4 *)(base + kOffSeeds);
  ma.sc = sc;
  ma.jobs = (JobRec *)(base + kOffJobs);
  ma.job_seq = seq;
  ma.job_ring = kNaRing;
  ma.W = nq;
  ma.cap = 0;
  ma.seg_count = (unsigned long long *)d_counts;
  ma.list = 0;
  ma.donate = 1;
  ma.timeout_cycles = 5000ll * (long long)(clk_khz > 0 ? clk_khz : 1965000);
  int per_sm = std::max(1, std::min(match_max_blocks_per_sm(), 4));
  launch_match(ma, std::max(sms, 1) * per_sm, s);
  if (cudaGetLastError() != cudaSuccess) return cuda_failed();

  unsigned int error = 0;
  if (cudaMemcpyAsync(&error, &sc->error, sizeof(error), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return cuda_failed();
  if (error & kErrTimeout) return done(DSM_ERR_TIMEOUT);
  if (error & kErrSeeds) return done(DSM_ERR_OVERFLOW);
  return done(DSM_OK);
}
