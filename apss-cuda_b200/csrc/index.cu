// Reference-semantics inverted index (cuapss_build_index): for every feature
// id f >= p of the caller's matrix (no remap), the rows containing f and
// their values, lists sorted by row, list pointers dim_ptr[d+1].
//
// Reference: generate_index_ptr4 (fengyilin118/APSS-CUDA
// similarity_search.cu:105-191) counts postings of ids >= 4096 per feature
// with global atomics; the host copies the counts back, scans them serially
// (1168-1186) and uploads dim_ptr; construct_Index2 (221-274) scatters
// (row, value) through atomicAdd cursors, leaving every list in
// nondeterministic order, and dim_ptr is re-uploaded (1256-1263) because the
// cursors consumed it. Here: posting counts and the exclusive scan stay on
// the device, and one stable LSD radix sort on (feature, row) places every
// posting, so each list is sorted by row and the build is deterministic.
#include <cuda_runtime.h>

#include <algorithm>

#include "index.cuh"
#include "prims.cuh"

namespace cuapss {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t work, int per_block) {
  int64_t g = ceil_div(std::max<int64_t>(work, 1), per_block);
  return (unsigned)std::min<int64_t>(g, 148 * 32);
}

// One warp per row: the entries with id >= p form a suffix of the sorted row.
__global__ void k_suffix_len(const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                             int64_t n, int32_t p, int64_t* __restrict__ start,
                             int64_t* __restrict__ len) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t lo = rp[i], hi = rp[i + 1];
    int cnt = 0;
    for (int64_t e = lo + lane; e < hi; e += 32) cnt += col[e] >= p;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) {
      start[i] = hi - cnt;
      len[i] = cnt;
    }
  }
}

__global__ void k_index_keys(const int64_t* __restrict__ start, const int64_t* __restrict__ len,
                             const int64_t* __restrict__ off, const int32_t* __restrict__ col,
                             int64_t n, int rbits, uint64_t* __restrict__ keys,
                             uint32_t* __restrict__ vals, int32_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t s = start[i], o = off[i];
    for (int64_t k = lane; k < len[i]; k += 32) {
      const int32_t f = col[s + k];
      keys[o + k] = ((uint64_t)f << rbits) | (uint64_t)i;
      vals[o + k] = (uint32_t)(s + k);
      atomicAdd(&counts[f], 1);
    }
  }
}

__global__ void k_index_fill(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             const float* __restrict__ val, int64_t T, uint64_t rmask,
                             int32_t* __restrict__ idx_row, float* __restrict__ idx_val) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < T;
       m += (int64_t)gridDim.x * blockDim.x) {
    idx_row[m] = (int32_t)(keys[m] & rmask);
    idx_val[m] = val[vals[m]];
  }
}

}  // namespace

cuapss_status build_ref_index(const int64_t* rp, const int32_t* col, const float* val, int64_t n,
                              int64_t d, int32_t p, int32_t* dim_ptr, int32_t** idx_row,
                              float** idx_val, int64_t* tail_nnz, Workspace& ws,
                              cudaStream_t st) {
  int64_t *start = nullptr, *len = nullptr, *off = nullptr;
  ST_TRY(ws.get("ri:start", (size_t)n + 1, &start));
  ST_TRY(ws.get("ri:len", (size_t)n + 1, &len));
  ST_TRY(ws.get("ri:off", (size_t)n + 1, &off));
  k_suffix_len<<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(rp, col, n, p, start, len);
  LAUNCH_CHECK();
  ST_TRY(exclusive_scan<int64_t>(len, off, n, off + n, ws, "ri:off", st));
  int64_t T = 0;
  CU_TRY(cudaMemcpyAsync(&T, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  *tail_nnz = T;
  uint64_t* keys = nullptr;
  uint32_t* vals = nullptr;
  int32_t* counts = nullptr;
  ST_TRY(ws.get("ri:keys", (size_t)T, &keys));
  ST_TRY(ws.get("ri:vals", (size_t)T, &vals));
  ST_TRY(ws.get("ri:counts", (size_t)d + 1, &counts));
  ST_TRY(ws.get("ri:row", (size_t)T, idx_row));
  ST_TRY(ws.get("ri:val", (size_t)T, idx_val));
  CU_TRY(cudaMemsetAsync(counts, 0, sizeof(int32_t) * (d + 1), st));
  const int rbits = std::max(1, bits_for((uint64_t)n));
  k_index_keys<<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(start, len, off, col, n, rbits,
                                                                keys, vals, counts);
  LAUNCH_CHECK();
  ST_TRY(radix_sort_pairs(keys, vals, T, rbits + std::max(1, bits_for((uint64_t)d)), ws, "ri", st));
  k_index_fill<<<grid_for(T, kThreads), kThreads, 0, st>>>(keys, vals, val, T, (1ull << rbits) - 1,
                                                          *idx_row, *idx_val);
  LAUNCH_CHECK();
  ST_TRY(exclusive_scan<int32_t>(counts, dim_ptr, d, dim_ptr + d, ws, "ri:dp", st));
  return CUAPSS_OK;
}

}  // namespace cuapss
