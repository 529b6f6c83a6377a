// Internal entry of the resident index shared with the request server
// (plain C++: no CUDA types).
#pragma once

#include <cstdint>

#include "cuapss.h"

namespace cuapss {

// cuapss_index_query that also reports the index rows the query was matched
// against (the rows that existed when it started).
cuapss_status index_query_rows(cuapss_ctx* ctx, const cuapss_index* idx, const cuapss_csr* q,
                               const float* t, cuapss_pairs* out, cuapss_stats* stats,
                               int64_t* rows_seen);

// cuapss_index_append in two parts: the new rows' segment, built and
// published (appends one at a time), and one merge of the trailing segments
// when the size policy calls for it (*merged: whether one ran; merges one at
// a time, concurrently with appends and queries). cuapss_index_append runs
// the first, then the second until no merge is due.
cuapss_status index_append_segment(cuapss_ctx* ctx, cuapss_index* idx, const cuapss_csr* x);
cuapss_status index_merge_step(cuapss_ctx* ctx, cuapss_index* idx, bool* merged);

}  // namespace cuapss
