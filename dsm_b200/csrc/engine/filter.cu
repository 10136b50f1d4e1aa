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

// LDF + NLF, one warp per data vertex (filter.cu:394-613): label equal,
// degree >= the query vertex's degree in the full query, and for every
// label l below the query's largest label + 1 at least as many neighbours
// of label l as the query vertex has.
__global__ void k_ldf_nlf(DevGraph g, const QFilterDesc *D, uint32_t *vcand, uint32_t *valid) {
  __shared__ uint32_t cnt[8][32];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nl = D->nlabels;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < g.nv; v += warps) {
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
      const uint32_t *run = adj_list(g, av);
      for (uint32_t i = lane; i < av.y; i += 32) {
        uint32_t l = g.lab[run[i] & kIdMask] & kLabelMask;
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
  }
}

// One op of the plan over every current candidate of its core vertex; a warp
// takes 32 vertices, then walks the candidates among them one by one with
// its lanes over the candidate's neighbours.
__global__ void k_filter_op(DevGraph g, const DevFilterOp *ops, uint32_t k, const uint32_t *vcand,
                            uint32_t *valid, uint32_t *enc, uint32_t words) {
  const DevFilterOp &op = ops[k];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t cu = op.core_u, pos = op.pos;
  for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < g.nv; base += warps * 32) {
    const uint32_t v = base + lane;
    const bool isc = v < g.nv && ((valid[v] >> cu) & 1u);
    for (uint32_t m = __ballot_sync(kFull, isc); m; m &= m - 1) {
      const uint32_t c = base + __ffs(m) - 1;
      // the candidate itself
      if (lane == 0) {
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
      // its neighbours
      const uint2 ac = g.adj[c];
      const uint32_t *run = adj_list(g, ac);
      for (uint32_t i = lane; i < ac.y; i += 32) {
        const uint32_t n = run[i] & kIdMask;
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
    }
  }
}

// compact (filter.cu:1692-1749): bitmap[u][v / 32] from the bit at u's
// position (or, with LDF+NLF only, from vcand).
__global__ void k_filter_compact(uint32_t nv, const QFilterDesc *D, const uint32_t *vcand, const uint32_t *enc,
                                 uint32_t words, uint32_t col_len, uint32_t *bitmap, int ldf_only) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < col_len; w += warps) {
    const uint32_t v = w * 32 + lane;
    for (uint32_t u = 0; u < D->nq; ++u) {
      bool b = false;
      if (v < nv) b = ldf_only ? ((vcand[v] >> u) & 1u) : ebit(enc, words, v, D->pos_of_u[u]);
      uint32_t m = __ballot_sync(kFull, b);
      if (lane == 0) bitmap[(size_t)u * col_len + w] = m;
    }
  }
}

}  // namespace

void launch_query_filter(const DevGraph &g, const FilterDevice &f, int mode, int num_sms, cudaStream_t s) {
  const int blocks = num_sms * 8;
  cudaMemsetAsync(f.enc, 0, (size_t)g.nv * f.words * 4, s);
  k_ldf_nlf<<<blocks, 256, 0, s>>>(g, f.desc, f.vcand, f.valid);
  if (mode >= 2)
    for (uint32_t k = 0; k < f.nops; ++k) k_filter_op<<<blocks, 256, 0, s>>>(g, f.ops, k, f.vcand, f.valid, f.enc, f.words);
  k_filter_compact<<<blocks, 256, 0, s>>>(g.nv, f.desc, f.vcand, f.enc, f.words, f.col_len, f.bitmap, mode < 2);
}

}  // namespace dsm
