// Reference-semantics inverted index build.
#pragma once

#include "common.cuh"

namespace cuapss {

// dim_ptr: device int32[d+1]. *idx_row / *idx_val receive workspace device
// arrays of *tail_nnz entries.
cuapss_status build_ref_index(const int64_t* rp, const int32_t* col, const float* val, int64_t n,
                              int64_t d, int32_t p, int32_t* dim_ptr, int32_t** idx_row,
                              float** idx_val, int64_t* tail_nnz, Workspace& ws,
                              cudaStream_t st);

}  // namespace cuapss
