// Context object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "cuapss.h"
#include "prep.cuh"
#include "side.cuh"

struct cuapss_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cuapss_opts opts{};
  int sms = 148;
  cuapss::Workspace ws;
  cudaEvent_t ev[6] = {};
  int64_t cand_cap = 0;
  // batched joins: the captured tile launches (updated in place when the
  // next batch has the same launch topology) and the tuner's choices
  cudaGraph_t batch_graph = nullptr;
  cudaGraphExec_t batch_exec = nullptr;
  std::map<uint64_t, int> tuned_p;
};

namespace cuapss {

struct DevCsr {
  int64_t n = 0, d = 0, nnz = 0;
  const int64_t* rp = nullptr;
  const int32_t* col = nullptr;
  const float* val = nullptr;
};

// Validates the descriptor and returns device pointers (staging host
// arrays into workspace buffers named by tag).
cuapss_status stage_csr(cuapss_ctx* ctx, const cuapss_csr* x, const std::string& tag,
                        DevCsr* out);

// The self-join (b == nullptr) or cross-join of staged matrices.
cuapss_status join_device(cuapss_ctx* ctx, const DevCsr& a, const DevCsr* b, float t,
                          cuapss_pairs* out, cuapss_stats* stats, int shard = 0,
                          int nshards = 1);

// Head width used when the options leave it to the library: n rows, nnz
// non-zeros over d features; prefix[k] = postings of the k most frequent
// features (rank_count_prefix; may be empty for FP32). Self-joins whose rare
// features are paired explicitly pass the first rank of those features and
// their postings (0: every tail feature is probed).
int choose_head_width(int precision, int64_t n, int64_t d, int64_t nnz,
                      const std::vector<int64_t>& prefix, int64_t rare_rank = 0,
                      int64_t rare_postings = 0);

// Whether the tile cost model puts the head at p at least twice the tail
// still probed (the tile kernel's two-J-block MMA tiles then pay).
bool head_bound_plan(int64_t p, int64_t n, int64_t nnz, const std::vector<int64_t>& prefix,
                     const RareCandidate& rare);

// Head width and rare-feature threshold of a self-join, chosen together by
// the tile cost model: the threshold (of cands, at most max_pairs pairs, or
// none) and p that minimise the modelled tile time plus the explicit pairs'
// cost. fixed_p > 0: that head width, the threshold alone is chosen.
// forced: the (single) candidate is taken whatever its modelled cost.
struct TilePlan {
  int p = 0;
  RareCandidate rare;  // max_count 0: no explicit pairs
};
TilePlan plan_tiles(int precision, int64_t n, int64_t d, int64_t nnz,
                    const std::vector<int64_t>& prefix,
                    const std::vector<RareCandidate>& cands, int64_t max_pairs, int fixed_p,
                    bool forced = false);

}  // namespace cuapss
