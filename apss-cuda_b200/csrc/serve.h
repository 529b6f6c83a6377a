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

}  // namespace cuapss
