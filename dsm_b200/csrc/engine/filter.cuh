// Device side of the cluster-encoding candidate filter.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace dsm {

// Per-query constants of the filter (full query: labels, degrees, neighbour
// label counts; plan: candidacy positions).
struct QFilterDesc {
  uint32_t nq;
  uint32_t nlabels;          // largest query label + 1 (copyMeta, io.cu:334)
  uint32_t label_us[32];     // per label: mask of query vertices carrying it
  uint32_t qdeg[16];
  uint32_t pos_of_u[16];
  uint8_t nlc[16][32];       // neighbour label counts of the full query
};

// One op of the plan (see host/query_plan.h FilterOp), compact form.
struct DevFilterOp {
  uint32_t kind, core_u, pos, nleaf;
  uint32_t leaf_u[16];
  uint32_t lp, rp, lcp, rcp;
  uint32_t comb_type, nsmall;
  uint32_t small_core_pos[32];
  uint32_t leaf_src_count[16];
  uint16_t leaf_src[16][32];
};

struct FilterDevice {
  const QFilterDesc *desc;
  const DevFilterOp *ops;
  uint32_t nops;
  uint32_t *vcand, *valid, *enc, *bitmap;
  uint32_t words, col_len;
};

// mode 1: LDF+NLF only; mode 2: cluster encoding.  Writes f.bitmap.
void launch_query_filter(const DevGraph &g, const FilterDevice &f, int mode, int num_sms, cudaStream_t s);

}  // namespace dsm
