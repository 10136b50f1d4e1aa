// Cluster-encoding candidate filter on the GPU (filter.cu of the reference:
// oneRoundFilterBidirectionKernel 394-613, encode/merge/combine 615-1177,
// compact 1692-1749), run per query on the batch's union graph.
//
// The graph's runs are label-major (entries carry the label slot above the
// id).  Layout per query: vcand[v] (bit u: v passes LDF+NLF for u, the
// reference's d_v_candidate_us_), valid[v] (bit u: v is still a candidate
// of u; merges and combines clear bits, as the reference overwrites entries
// of its per-u candidate lists), enc[v * words + pos / 32] (cluster
// encodings), bitmap[u * col_len + v / 32] (per-u result, the reference's
// compact layout).  Ops run in the host plan's order, one launch each; inside
// an op the bits read belong to older clusters and the bits written to the
// op's own cluster, and every write is an atomic OR / AND, so the result does
// not depend on thread order (the reference's plain read-modify-writes next
// to atomicOr, filter.cu:688/763/868/874, can lose bits; this is their
// race-free intent).
//
// Incremental runs.  The reference recomputes the whole filter every batch
// (main.cu:213).  Here a query's state stays resident between batches, and a
// batch recomputes only the vertices whose state can differ from the previous
// batch's: the union graphs of two batches differ only in edges at endpoints
// of the two batches' updates (T), LDF+NLF of a vertex depends on its own
// adjacency, and each op moves information one hop (a core candidate's
// validity to its neighbours' leaf bits), so after D ops only vertices within
// D hops of T can differ.  For those (the region) every op is recomputed in
// pull form: a receiver takes an op's leaf bits if some neighbour is a valid
// core candidate at the op's start.  A neighbour inside the region has that
// validity in `valid` as the run proceeds; one outside kept its whole history,
// so its validity at op k is replayed from its final bits (its LDF+NLF bit and
// the checks of the merges and combines before k with the same core, which
// read bits of earlier layers that nothing rewrites later).  A region that
// outgrows its list, a state not computed in the previous batch, or a graph
// changed outside a filtered batch make the run recompute every vertex.
#include "filter.cuh"

namespace dsm {

namespace {

__device__ __forceinline__ bool ebit(const uint32_t *enc, uint32_t words, uint32_t v, uint32_t pos) {
  return (enc[(size_t)v * words + (pos >> 5)] >> (pos & 31)) & 1u;
}
__device__ __forceinline__ void eset(uint32_t *enc, uint32_t words, uint32_t v, uint32_t pos) {
  atomicOr(&enc[(size_t)v * words + (pos >> 5)], 1u << (pos & 31));
}
__device__ __forceinline__ void eclr(uint32_t *enc, uint32_t words, uint32_t v, uint32_t pos) {
  atomicAnd(&enc[(size_t)v * words + (pos >> 5)], ~(1u << (pos & 31)));
}

// Whether this run of the query recomputes every vertex.
__device__ __forceinline__ bool decide_full(const QFilterDesc *D, const RegionDevice &rg, int force_full) {
  if (force_full || rg.info == nullptr) return true;
  const RegionInfo &I = *rg.info;
  if (I.stale_now || I.prev_ov || D->hops > I.hops || I.ov_round <= D->hops) return true;
  return D->fepoch + 1 != I.epoch;  // not computed in the previous filtered batch
}

// The vertices of this run: all of them, or the query's region.
struct Scope {
  bool full;
  uint32_t count;
  const uint32_t *list;
};
__device__ __forceinline__ Scope scope_of(const QFilterDesc *D, const RegionDevice &rg, uint32_t nv) {
  Scope s;
  s.full = D->full_now != 0;
  s.list = rg.list;
  s.count = s.full ? nv : rg.info->bound[D->hops];
  return s;
}

__device__ __forceinline__ bool in_region(const RegionDevice &rg, uint32_t epoch, uint32_t hops, uint32_t v) {
  const uint32_t m = rg.mark[v];
  return (m >> 6) == epoch && (m & 63) <= hops;
}

// LDF + NLF, one warp per data vertex (filter.cu:394-613): label equal,
// degree >= the query vertex's degree in the full query, and for every
// label l below the query's largest label + 1 at least as many neighbours
// of label l as the query vertex has.  Clears the vertex's encodings.  The
// first kernel of a run: decides whether the run is full.
__global__ void k_ldf_nlf(DevGraph g, QFilterDesc *D, uint32_t *vcand, uint32_t *valid, uint32_t *enc,
                          uint32_t words, RegionDevice rg, int force_full) {
  __shared__ uint32_t cnt[8][32];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nl = D->nlabels;
  const bool full = decide_full(D, rg, force_full);
  if (blockIdx.x == 0 && threadIdx.x == 0) D->full_now = full ? 1u : 0u;
  const uint32_t count = full ? g.nv : rg.info->bound[D->hops];
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warps) {
    const uint32_t v = full ? i : rg.list[i];
    const uint32_t lv = g.lab[v] & kLabelMask;
    const uint2 av = g.adj[v];
    uint32_t um = lv < nl ? D->label_us[lv] : 0u;  // query vertices with this label
    uint32_t keep = 0;
    for (uint32_t b = um; b; b &= b - 1) {
      uint32_t u = __ffs(b) - 1;
      if (D->qdeg[u] <= av.y) keep |= 1u << u;
    }
    uint32_t res = 0;
    if (keep) {
      cnt[wib][lane] = 0;
      __syncwarp();
      // the run starts on a 16-byte boundary: four entries per lane per load
      const uint32_t *run = adj_list(g, av);
      const uint4 *run4 = reinterpret_cast<const uint4 *>(run);
      const uint32_t n4 = av.y >> 2;
      for (uint32_t k = lane; k < n4; k += 32) {
        const uint4 q = run4[k];
        const uint32_t e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const uint32_t l = g.lab[e[t] & kIdMask] & kLabelMask;
          if (l < nl) atomicAdd(&cnt[wib][l], 1u);
        }
      }
      for (uint32_t k = 4 * n4 + lane; k < av.y; k += 32) {
        const uint32_t l = g.lab[run[k] & kIdMask] & kLabelMask;
        if (l < nl) atomicAdd(&cnt[wib][l], 1u);
      }
      __syncwarp();
      const uint32_t mine = cnt[wib][lane];
      for (uint32_t b = keep; b; b &= b - 1) {
        uint32_t u = __ffs(b) - 1;
        bool pass = lane >= nl || mine >= D->nlc[u][lane];
        if (__all_sync(kFull, pass)) res |= 1u << u;
      }
      __syncwarp();
    }
    if (lane == 0) {
      vcand[v] = res;
      valid[v] = res;
    }
    for (uint32_t w = lane; w < words; w += 32) enc[(size_t)v * words + w] = 0;
  }
}

// The core rule of op k for candidate c (valid for the op's core at its start).
__device__ __forceinline__ void core_rule(const DevFilterOp &op, uint32_t c, uint32_t *valid, uint32_t *enc,
                                          uint32_t words) {
  const uint32_t cu = op.core_u, pos = op.pos;
  if (op.kind == 0) {  // encodeKernel: core bit
    eset(enc, words, c, pos);
  } else if (op.kind == 1) {  // mergeKernel: both parents' bits of the core
    if (ebit(enc, words, c, op.lp) && ebit(enc, words, c, op.rp)) eset(enc, words, c, pos);
    else atomicAnd(&valid[c], ~(1u << cu));
  } else {  // combineMultipleClustersKernel: every small cluster's core bit
    bool all = true;
    for (uint32_t s = 0; s < op.nsmall; ++s) all = all && ebit(enc, words, c, op.small_core_pos[s]);
    if (all) {
      if (op.comb_type == 0) eset(enc, words, c, pos);
    } else {
      eclr(enc, words, c, pos);
      atomicAnd(&valid[c], ~(1u << cu));
    }
  }
}

// The leaf rule of op k for receiver n (a neighbour of a valid core candidate).
__device__ __forceinline__ void leaf_rule(const DevFilterOp &op, uint32_t n, const uint32_t *vcand, uint32_t *enc,
                                          uint32_t words) {
  const uint32_t pos = op.pos;
  if (op.kind == 0) {
    const uint32_t code = vcand[n];
    for (uint32_t j = 0; j < op.nleaf; ++j)
      if ((code >> op.leaf_u[j]) & 1u) eset(enc, words, n, pos + 1 + j);
  } else if (op.kind == 1) {
    if (ebit(enc, words, n, op.lcp)) eset(enc, words, n, pos + 1);
    if (op.rcp != op.rp && ebit(enc, words, n, op.rcp)) eset(enc, words, n, pos + 2);
  } else {
    for (uint32_t j = 0; j < op.nleaf; ++j) {
      bool fv = true;
      for (uint32_t t = 0; t < op.leaf_src_count[j]; ++t) fv = fv && ebit(enc, words, n, op.leaf_src[j][t]);
      if (op.comb_type == 1) {
        if (!fv) eclr(enc, words, n, pos + 1 + j);
      } else if (fv) {
        eset(enc, words, n, pos + 1 + j);
      }
    }
  }
}

// Full runs: one op over every current candidate of its core vertex; a warp
// takes 32 vertices, then walks the candidates among them one by one with
// its lanes over the candidate's neighbours.
__global__ void k_filter_op(DevGraph g, const QFilterDesc *D, const DevFilterOp *ops, uint32_t k,
                            const uint32_t *vcand, uint32_t *valid, uint32_t *enc, uint32_t words) {
  if (!D->full_now) return;
  const DevFilterOp &op = ops[k];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t cu = op.core_u;
  for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < g.nv; base += warps * 32) {
    const uint32_t v = base + lane;
    const bool isc = v < g.nv && ((valid[v] >> cu) & 1u);
    for (uint32_t m = __ballot_sync(kFull, isc); m; m &= m - 1) {
      const uint32_t c = base + __ffs(m) - 1;
      if (lane == 0) core_rule(op, c, valid, enc, words);
      // its neighbours
      const uint2 ac = g.adj[c];
      const uint32_t *run = adj_list(g, ac);
      for (uint32_t i = lane; i < ac.y; i += 32) leaf_rule(op, run[i] & kIdMask, vcand, enc, words);
    }
  }
}

// Validity of c for the core of op k at the op's start, for a vertex outside
// the region (its bits are those of the previous run, which it shares).
__device__ __forceinline__ bool replayed_valid(const DevFilterOp *ops, const DevFilterOp &op, uint32_t c,
                                               const uint32_t *vcand, const uint32_t *enc, uint32_t words) {
  if (!((vcand[c] >> op.core_u) & 1u)) return false;
  for (uint32_t p = 0; p < op.nprior; ++p) {
    const DevFilterOp &q = ops[op.prior[p]];
    if (q.kind == 1) {
      if (!(ebit(enc, words, c, q.lp) && ebit(enc, words, c, q.rp))) return false;
    } else {
      for (uint32_t s = 0; s < q.nsmall; ++s)
        if (!ebit(enc, words, c, q.small_core_pos[s])) return false;
    }
  }
  return true;
}

// Region runs, op k, first half: every receiver of the region pulls its
// leaf bits (a warp per receiver scans its neighbours for a valid core
// candidate at the op's start).
__global__ void k_filter_pull(DevGraph g, const QFilterDesc *D, const DevFilterOp *ops, uint32_t k,
                              const uint32_t *vcand, const uint32_t *valid, uint32_t *enc, uint32_t words,
                              RegionDevice rg) {
  if (D->full_now) return;
  const DevFilterOp &op = ops[k];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t epoch = rg.info->epoch, hops = D->hops;
  const uint32_t count = rg.info->bound[hops];
  const uint32_t cu = op.core_u;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warps) {
    const uint32_t n = rg.list[i];
    const uint2 an = g.adj[n];
    const uint32_t *run = adj_list(g, an);
    bool has = false;
    for (uint32_t b = 0; b < an.y && !has; b += 32) {
      bool cv = false;
      if (b + lane < an.y) {
        const uint32_t c = run[b + lane] & kIdMask;
        cv = in_region(rg, epoch, hops, c) ? ((valid[c] >> cu) & 1u) != 0
                                           : replayed_valid(ops, op, c, vcand, enc, words);
      }
      has = __any_sync(kFull, cv);
    }
    if (has && lane == 0) leaf_rule(op, n, vcand, enc, words);
  }
}

// Region runs, op k, second half: the core rule for the region's candidates.
__global__ void k_filter_core(const QFilterDesc *D, const DevFilterOp *ops, uint32_t k, uint32_t *valid,
                              uint32_t *enc, uint32_t words, RegionDevice rg) {
  if (D->full_now) return;
  const DevFilterOp &op = ops[k];
  const uint32_t count = rg.info->bound[D->hops];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t c = rg.list[i];
    if ((valid[c] >> op.core_u) & 1u) core_rule(op, c, valid, enc, words);
  }
}

// compact (filter.cu:1692-1749): bitmap[u][v / 32] from the bit at u's
// position (or, with LDF+NLF only, from vcand).  Full runs: a warp per word;
// region runs: a warp per region vertex, rewriting its whole word.  The
// last kernel of a run: records the epoch the state belongs to.
__global__ void k_filter_compact(uint32_t nv, QFilterDesc *D, const uint32_t *vcand, const uint32_t *enc,
                                 uint32_t words, uint32_t col_len, uint32_t *bitmap, int ldf_only, RegionDevice rg) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const Scope sc = scope_of(D, rg, nv);
  const uint32_t count = sc.full ? col_len : sc.count;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warps) {
    const uint32_t w = sc.full ? i : (sc.list[i] >> 5);
    const uint32_t v = w * 32 + lane;
    for (uint32_t u = 0; u < D->nq; ++u) {
      bool b = false;
      if (v < nv) b = ldf_only ? ((vcand[v] >> u) & 1u) : ebit(enc, words, v, D->pos_of_u[u]);
      uint32_t m = __ballot_sync(kFull, b);
      if (lane == 0) bitmap[(size_t)u * col_len + w] = m;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) D->fepoch = rg.info ? rg.info->epoch : 0xFFFFFFFFu;
}

// ---- region ----------------------------------------------------------------
__device__ __forceinline__ void claim(const RegionDevice &rg, uint32_t epoch, uint32_t v, uint32_t hop) {
  const uint32_t old = rg.mark[v];
  if ((old >> 6) == epoch) return;
  if (atomicCAS(&rg.mark[v], old, (epoch << 6) | hop) != old) return;  // claimed by another thread
  const uint32_t idx = atomicAdd(&rg.info->total, 1u);
  if (idx < rg.info->cap) rg.list[idx] = v;
  else atomicMin(&rg.info->ov_round, hop);
}

__global__ void k_region_begin(RegionInfo *I, uint32_t hops) {
  I->stale_now = I->stale;
  I->stale = 0;
  I->epoch = (I->epoch + 1) & 0x03FFFFFFu;
  if (I->epoch == 0) I->epoch = 1;
  I->total = 0;
  I->ov_round = 64;
  I->hops = hops;
}

__global__ void k_region_seed(DevGraph g, RegionDevice rg, const uint32_t *hdr_n, const uint4 *upd) {
  const uint32_t n = *hdr_n, epoch = rg.info->epoch, np = rg.info->prev_cnt;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * n + np; i += gridDim.x * blockDim.x) {
    uint32_t v;
    if (i < 2 * n) {
      const uint4 u = upd[i >> 1];
      v = (i & 1) ? u.z : u.y;
    } else {
      v = rg.prev[i - 2 * n];
    }
    if (v < g.nv) claim(rg, epoch, v, 0);
  }
}

__global__ void k_region_close(RegionInfo *I, uint32_t hop) { I->bound[hop] = min(I->total, I->cap); }

// Hop `hop`: every neighbour of the vertices first reached at hop - 1.
__global__ void k_region_expand(DevGraph g, RegionDevice rg, uint32_t hop) {
  const RegionInfo &I = *rg.info;
  if (I.ov_round < 64) return;  // the list is full: queries that far out run in full
  const uint32_t lo = hop >= 2 ? I.bound[hop - 2] : 0u, hi = I.bound[hop - 1];
  const uint32_t lane = threadIdx.x & 31, epoch = I.epoch;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < hi; i += warps) {
    const uint32_t v = rg.list[i];
    const uint2 av = g.adj[v];
    const uint32_t *run = adj_list(g, av);
    const uint4 *run4 = reinterpret_cast<const uint4 *>(run);  // 16-byte aligned run
    const uint32_t n4 = av.y >> 2;
    for (uint32_t k = lane; k < n4; k += 32) {
      const uint4 q = run4[k];
      claim(rg, epoch, q.x & kIdMask, hop);
      claim(rg, epoch, q.y & kIdMask, hop);
      claim(rg, epoch, q.z & kIdMask, hop);
      claim(rg, epoch, q.w & kIdMask, hop);
    }
    for (uint32_t k = 4 * n4 + lane; k < av.y; k += 32) claim(rg, epoch, run[k] & kIdMask, hop);
    if (*(volatile const uint32_t *)&rg.info->ov_round < 64) return;
  }
}

// The batch's endpoints become the next batch's previous endpoints.
__global__ void k_region_save(RegionDevice rg, const uint32_t *hdr_n, const uint4 *upd) {
  const uint32_t n = *hdr_n, cap = rg.info->prev_cap;
  const bool fits = 2ull * n <= cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n && fits; i += gridDim.x * blockDim.x) {
    const uint4 u = upd[i];
    rg.prev[2 * i] = u.y;
    rg.prev[2 * i + 1] = u.z;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    rg.info->prev_cnt = fits ? 2 * n : 0u;
    rg.info->prev_ov = fits ? 0u : 1u;
  }
}

}  // namespace

void launch_query_filter(const DevGraph &g, const FilterDevice &f, int mode, int num_sms, cudaStream_t s,
                         const RegionDevice &rg, int force_full) {
  const int blocks = num_sms * 8;
  QFilterDesc *D = const_cast<QFilterDesc *>(f.desc);
  k_ldf_nlf<<<blocks, 256, 0, s>>>(g, D, f.vcand, f.valid, f.enc, f.words, rg, force_full);
  if (mode >= 2)
    for (uint32_t k = 0; k < f.nops; ++k) {
      k_filter_op<<<blocks, 256, 0, s>>>(g, D, f.ops, k, f.vcand, f.valid, f.enc, f.words);
      if (rg.info) {
        k_filter_pull<<<blocks, 256, 0, s>>>(g, D, f.ops, k, f.vcand, f.valid, f.enc, f.words, rg);
        k_filter_core<<<blocks, 256, 0, s>>>(D, f.ops, k, f.valid, f.enc, f.words, rg);
      }
    }
  k_filter_compact<<<blocks, 256, 0, s>>>(g.nv, D, f.vcand, f.enc, f.words, f.col_len, f.bitmap, mode < 2, rg);
}

void launch_region_build(const DevGraph &g, const RegionDevice &rg, const uint32_t *hdr_n, const uint4 *upd,
                         uint32_t hops, int num_sms, cudaStream_t s) {
  k_region_begin<<<1, 1, 0, s>>>(rg.info, hops);
  k_region_seed<<<num_sms * 4, 256, 0, s>>>(g, rg, hdr_n, upd);
  k_region_close<<<1, 1, 0, s>>>(rg.info, 0);
  for (uint32_t h = 1; h <= hops; ++h) {
    k_region_expand<<<num_sms * 8, 256, 0, s>>>(g, rg, h);
    k_region_close<<<1, 1, 0, s>>>(rg.info, h);
  }
}

void launch_region_save(const RegionDevice &rg, const uint32_t *hdr_n, const uint4 *upd, cudaStream_t s) {
  k_region_save<<<64, 256, 0, s>>>(rg, hdr_n, upd);
}

}  // namespace dsm
