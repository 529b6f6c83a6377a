// Device primitives: exclusive scan and LSD radix sort of (u64 key, u32 value)
// pairs. Hand-written for sm_100a; used by the index build, the frequency
// remap and the output sort.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "common.cuh"

namespace cuapss {

// ---------------------------------------------------------------- scan ----
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
template <typename T, int NT>
__device__ __forceinline__ T block_excl_scan(T v, T* total) {
  __shared__ T warp_sums[NT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T inc = warp_incl_scan(v);
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  if (w == 0) {
    T s = lane < NT / 32 ? warp_sums[lane] : T(0);
    s = warp_incl_scan(s);
    if (lane < NT / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  T before = w > 0 ? warp_sums[w - 1] : T(0);
  *total = warp_sums[NT / 32 - 1];
  __syncthreads();
  return before + inc - v;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const T* __restrict__ in, int64_t n,
                                                              T* __restrict__ partial) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  T tot;
  block_excl_scan<T, kScanThreads>(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const T* __restrict__ in, T* __restrict__ out,
                                                             int64_t n, const T* __restrict__ offsets,
                                                             T* __restrict__ total) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;  // blocked
    v[k] = i < n ? in[i] : T(0);
    s += v[k];
  }
  T tot;
  T run = block_excl_scan<T, kScanThreads>(s, &tot);
  if (offsets) run += offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total = run;
}

// Exclusive scan of in[0..n) into out[0..n) (may alias). If total != nullptr
// the sum is written to *total (device pointer). `tag` names workspace.
template <typename T>
cuapss_status exclusive_scan(const T* in, T* out, int64_t n, T* total, Workspace& ws,
                             const std::string& tag, cudaStream_t st, int level = 0) {
  if (n <= 0) {
    if (total) CU_TRY(cudaMemsetAsync(total, 0, sizeof(T), st));
    return CUAPSS_OK;
  }
  const int64_t nb = ceil_div(n, kScanTile);
  if (nb == 1) {
    k_scan_apply<T><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, total);
    LAUNCH_CHECK();
    return CUAPSS_OK;
  }
  T* partial = nullptr;
  ST_TRY(ws.get(tag + ":scan" + std::to_string(level), (size_t)nb, &partial));
  k_scan_reduce<T><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, partial);
  LAUNCH_CHECK();
  ST_TRY(exclusive_scan<T>(partial, partial, nb, (T*)nullptr, ws, tag, st, level + 1));
  k_scan_apply<T><<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, partial, total);
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

// ---------------------------------------------------------- radix sort ----
constexpr int kRsWarps = 8;
constexpr int kRsChunks = 8;
constexpr int kRsThreads = kRsWarps * 32;
constexpr int kRsTile = kRsWarps * kRsChunks * 32;  // 2048

static __global__ void __launch_bounds__(kRsThreads) k_rs_upsweep(const uint64_t* __restrict__ keys, int64_t n,
                                                           int shift, uint32_t* __restrict__ hist,
                                                           int nblocks) {
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int i = threadIdx.x; i < kRsTile; i += kRsThreads) {
    const int64_t idx = base + i;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter: elements of a tile are ranked in index order (warp w owns
// elements [w*256, w*256+256) of the tile, in chunks of 32 lanes), placed in
// shared memory in digit order, then written out so that consecutive threads
// write consecutive addresses of each digit's run (coalesced stores).
static __global__ void __launch_bounds__(kRsThreads) k_rs_downsweep(const uint64_t* __restrict__ kin,
                                                             const uint32_t* __restrict__ vin,
                                                             uint64_t* __restrict__ kout,
                                                             uint32_t* __restrict__ vout, int64_t n,
                                                             int shift, const uint32_t* __restrict__ offs,
                                                             int nblocks) {
  __shared__ uint32_t wcnt[kRsWarps][256];
  __shared__ uint32_t dstart[256];  // first tile slot of each digit
  __shared__ uint32_t dglob[256];   // first output position of each digit for this tile
  __shared__ uint32_t wsum[kRsWarps];
  __shared__ uint64_t skey[kRsTile];
  __shared__ uint32_t sval[kRsTile];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kRsWarps * 256; i += kRsThreads) (&wcnt[0][0])[i] = 0;
  dglob[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
  __syncthreads();
  const int64_t tile0 = (int64_t)blockIdx.x * kRsTile;
  const int64_t base = tile0 + (int64_t)w * (kRsChunks * 32);
  uint64_t key[kRsChunks];
  uint32_t val[kRsChunks];
  uint32_t rank[kRsChunks];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int c = 0; c < kRsChunks; ++c) {
    const int64_t idx = base + c * 32 + lane;
    const bool valid = idx < n;
    key[c] = valid ? kin[idx] : 0ull;
    val[c] = valid ? vin[idx] : 0u;
    const unsigned d = (unsigned)(key[c] >> shift) & 255u;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    uint32_t before = 0, peers = 0;
    if (valid) {
      peers = __match_any_sync(vmask, d);
      before = wcnt[w][d];
    }
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wcnt[w][d] = before + __popc(peers);
    __syncwarp();
    rank[c] = before + __popc(peers & lt);
  }
  __syncthreads();
  {
    // per digit: offsets of the warps inside the digit, then the tile's
    // exclusive scan over digits (kRsThreads == 256 digits)
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kRsWarps; ++ww) {
      const uint32_t t = wcnt[ww][d];
      wcnt[ww][d] = run;
      run += t;
    }
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t before = 0;
    for (int ww = 0; ww < w; ++ww) before += wsum[ww];
    dstart[d] = before + x - run;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < kRsChunks; ++c) {
    const int64_t idx = base + c * 32 + lane;
    if (idx < n) {
      const unsigned d = (unsigned)(key[c] >> shift) & 255u;
      const uint32_t lp = dstart[d] + wcnt[w][d] + rank[c];
      skey[lp] = key[c];
      sval[lp] = val[c];
    }
  }
  __syncthreads();
  const int tile_n = (int)(n - tile0 < kRsTile ? n - tile0 : kRsTile);
  for (int i = threadIdx.x; i < tile_n; i += kRsThreads) {
    const uint64_t k = skey[i];
    const unsigned d = (unsigned)(k >> shift) & 255u;
    const int64_t pos = (int64_t)dglob[d] + (i - (int)dstart[d]);
    kout[pos] = k;
    vout[pos] = sval[i];
  }
}

// Sorts (keys, vals) in place by keys' bits [0, nbits), stable.
inline cuapss_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, int nbits,
                                      Workspace& ws, const std::string& tag, cudaStream_t st) {
  if (n <= 1 || nbits <= 0) return CUAPSS_OK;
  if (n >= (int64_t)UINT32_MAX) return CUAPSS_EINVAL;
  const int nblocks = (int)ceil_div(n, kRsTile);
  uint64_t* k2 = nullptr;
  uint32_t* v2 = nullptr;
  uint32_t* hist = nullptr;
  ST_TRY(ws.get(tag + ":rs_k", (size_t)n, &k2));
  ST_TRY(ws.get(tag + ":rs_v", (size_t)n, &v2));
  ST_TRY(ws.get(tag + ":rs_h", (size_t)nblocks * 256 + 1, &hist));
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = k2;
  uint32_t* vb = v2;
  int passes = 0;
  for (int shift = 0; shift < nbits; shift += 8, ++passes) {
    k_rs_upsweep<<<nblocks, kRsThreads, 0, st>>>(ka, n, shift, hist, nblocks);
    LAUNCH_CHECK();
    ST_TRY(exclusive_scan<uint32_t>(hist, hist, (int64_t)nblocks * 256, nullptr, ws, tag + ":rs", st));
    k_rs_downsweep<<<nblocks, kRsThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist, nblocks);
    LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (passes & 1) {
    CU_TRY(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, st));
    CU_TRY(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  }
  return CUAPSS_OK;
}


}  // namespace cuapss
