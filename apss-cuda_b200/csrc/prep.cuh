// Preparation of one join operand: validation, frequency remap, head block
// and inverted lists (rows keep the caller's order).
#pragma once

#include <string>
#include <vector>

#include "common.cuh"
#include "side.cuh"

namespace cuapss {

struct PrepOptions {
  int p = 64;           // head width (multiple of 32 for the FP32 head block)
  int want_head32 = 1;  // build the FP32 head block
  int want_head16 = 0;  // build the BF16 head block
  int want_csc = 0;     // build the global inverted lists (cptr/csc)
  int balance_rows = 0; // deal rows into blocks by tail non-zeros (rowperm); else caller order
  // Self-joins: features of rank >= rare_from (each occurring in at most
  // rare_max_count rows) are paired explicitly instead of probed; 0: off.
  int64_t rare_from = 0;
  int rare_max_count = 0;
  // Row-block shard of a self-join: only the explicit pairs of the tiles
  // (I, J) with I % rare_nshards == rare_shard are built.
  int rare_shard = 0;
  int rare_nshards = 1;
};

// Validates a device CSR. counts (device, d entries, may be null) are
// incremented per posting. *nrm_max receives the largest row norm.
cuapss_status validate_csr(const int64_t* rp, const int32_t* col, const float* val, int64_t n,
                           int64_t d, int64_t nnz, float tol, int check, int32_t* counts,
                           double* nrm_max, Workspace& ws, const std::string& tag,
                           cudaStream_t st);

// perm[f] = rank of feature f by (count desc, id asc); identity if !remap.
cuapss_status feature_perm(const int32_t* counts, int64_t d, int64_t max_count, int remap,
                           int32_t* perm, Workspace& ws, cudaStream_t st);

// Host prefix sums of the posting counts in rank order, after feature_perm:
// (*prefix)[k] = postings of the k most frequent features, k = 0 .. min(m, d).
cuapss_status rank_count_prefix(const int32_t* counts, int64_t d, int remap, int64_t m,
                                Workspace& ws, cudaStream_t st, std::vector<int64_t>* prefix);

// Rare features of a self-join (explicit pairs instead of probes), for each
// threshold C in {2048, 1024, ..., 16}: the features occurring in at most C
// rows, which under the frequency remap hold the ranks from `rank` on, their
// postings and their pairs. Thresholds with no such feature are left out.
constexpr int kMaxRareCount = 2048;
struct RareCandidate {
  int max_count = 0;      // C
  int64_t rank = 0;       // first rank of the features with count <= C
  int64_t pairs = 0;      // sum of count (count - 1) / 2 over them
  int64_t postings = 0;   // sum of count over them
};
cuapss_status rare_feature_candidates(const int32_t* counts, int64_t d, Workspace& ws,
                                      cudaStream_t st, std::vector<RareCandidate>* cands);

// Builds every array of `s` (s.rp0/col0/val0/n/d/nnz must be set).
cuapss_status build_side(Side& s, const PrepOptions& o, const int32_t* perm, Workspace& ws,
                         const std::string& tag, cudaStream_t st);


}  // namespace cuapss
