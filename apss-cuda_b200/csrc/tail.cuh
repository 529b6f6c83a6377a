// Tail phase shared by the pair-tile kernels: the sparse, feature-parallel
// part of the hybrid similarity.
//
// Both sides use block-local inverted lists (the tail postings of one
// 128-row block sorted by feature). For a unit's I block, its feature groups
// (sorted feature, first posting) and postings (row in block, value) are
// staged once in shared memory, with a direct table for the most frequent
// tail features. For every tile (I, J), each posting (c, f, v) of the J
// block's list finds the I group of f (table or binary search); every I
// posting (r, u) of that group adds u * v into the shared-memory accumulator
// acc[r][c] with a shared-memory atomic. The accumulator is fixed point
// (kTailScale = 2^30 per unit): each FP32 product is rounded to the 2^-30
// grid and integer atomics sum exactly, in any order, so the tail is
// deterministic and its error is the product rounding plus 2^-31 per term.
// This replaces the reference's per-feature block schedule and its
// global-memory atomics into a dense n x n array (fengyilin118/APSS-CUDA
// generate_auxiliary_variable{,2}{,_apss} and similarity_join1 /
// similarity_apss1, similarity_search.cu:323-437 and 577-735).
#pragma once

#include "tiles.cuh"

namespace cuapss {

// Tail features below kWarm (the most frequent ones after the head) are
// looked up in a direct table; the rest by binary search.
constexpr int kWarm = 2048;
constexpr float kTailScale = 1073741824.0f;     // 2^30
constexpr float kTailUnscale = 9.313225746154785e-10f;  // 2^-30

__device__ __forceinline__ int tail_fixed(float prod) {
  return __float2int_rn(prod * kTailScale);
}
constexpr uint16_t kNoGroup = 0xffff;

// I side of the match: generic pointers (shared memory when the block fits
// the staging capacity, the global arrays otherwise).
struct TailI {
  const uint32_t* gf;  // [G] feature of each group, ascending
  const uint32_t* gs;  // [G+1] first posting of each group
  const uint8_t* er;   // posting: row in block
  const float* eu;     // posting: value
  const uint16_t* warm;  // [kWarm] group of warm feature f, or kNoGroup
  int G;
  int gw;              // groups with a warm feature (a prefix of gf)
};

// Stage I block `I` into shared memory if it fits (returns the view either
// way). All NT threads call it; a __syncthreads() must follow before use.
template <int NT>
__device__ __forceinline__ TailI stage_tail_i(const TileArgs& A, int I, uint32_t* s_gf,
                                              uint32_t* s_gs, uint8_t* s_er, float* s_eu,
                                              uint16_t* s_warm, int gcap, int ecap) {
  const int64_t g0 = A.gptrI[I], g1 = A.gptrI[I + 1];
  const int64_t e0 = A.gstartI[g0];
  const int64_t e1 = A.gstartI[g1];
  TailI v;
  v.G = (int)(g1 - g0);
  for (int w = threadIdx.x; w < kWarm; w += NT) s_warm[w] = kNoGroup;
  __syncthreads();
  int gw = 0;
  {
    // groups are sorted by feature: the warm ones form a prefix
    int lo = 0, hi = v.G;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (A.gfeatI[g0 + mid] < (uint32_t)kWarm) lo = mid + 1;
      else hi = mid;
    }
    gw = lo;
  }
  for (int g = threadIdx.x; g < gw; g += NT) s_warm[A.gfeatI[g0 + g]] = (uint16_t)g;
  v.gw = gw;
  v.warm = s_warm;
  if (g1 - g0 <= gcap && e1 - e0 <= ecap) {
    for (int64_t g = threadIdx.x; g < g1 - g0; g += NT) {
      s_gf[g] = A.gfeatI[g0 + g];
      s_gs[g] = A.gstartI[g0 + g] - (uint32_t)e0;
    }
    if (threadIdx.x == 0) s_gs[g1 - g0] = (uint32_t)(e1 - e0);
    for (int64_t e = threadIdx.x; e < e1 - e0; e += NT) {
      s_er[e] = A.bilI_r[e0 + e];
      s_eu[e] = A.bilI_u[e0 + e];
    }
    v.gf = s_gf;
    v.gs = s_gs;
    v.er = s_er;
    v.eu = s_eu;
  } else {
    v.gf = A.gfeatI + g0;
    v.gs = A.gstartI + g0;
    v.er = A.bilI_r;
    v.eu = A.bilI_u;
  }
  return v;
}

// Group of feature f in the I block, or -1.
__device__ __forceinline__ int find_group(const TailI& T, uint32_t f) {
  if (f < (uint32_t)kWarm) {
    const uint16_t g = T.warm[f];
    return g == kNoGroup ? -1 : (int)g;
  }
  int lo = T.gw, hi = T.G;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (T.gf[mid] < f) lo = mid + 1;
    else hi = mid;
  }
  return (lo < T.G && T.gf[lo] == f) ? lo : -1;
}

// Tail contributions of tile (I, J) into acc (row stride ld), computed by
// thread `tid` of `nthreads` cooperating threads. Postings are taken with a
// stride of nthreads so that the postings of one frequent feature (adjacent
// in the sorted list) go to adjacent lanes; each thread loads kTailBatch
// postings before matching them, to keep that many loads in flight.
constexpr int kTailBatch = 8;

__device__ __forceinline__ void tail_tile(const TileArgs& A, const TailI& T, int J, int* acc,
                                          int ld, int tid, int nthreads) {
  const int64_t k0 = A.bptrJ[J], k1 = A.bptrJ[J + 1];
  if (T.G <= 0) return;
  for (int64_t kb = k0 + tid; kb < k1; kb += (int64_t)kTailBatch * nthreads) {
    uint2 rec[kTailBatch];
#pragma unroll
    for (int q = 0; q < kTailBatch; ++q) {
      const int64_t k = kb + (int64_t)q * nthreads;
      rec[q] = k < k1 ? __ldg(&A.bilJ_rec[k]) : make_uint2(0xffffffffu, 0u);
    }
#pragma unroll
    for (int q = 0; q < kTailBatch; ++q) {
      if (rec[q].x == 0xffffffffu) continue;
      const int g = find_group(T, rec[q].x >> 8);
      if (g >= 0) {
        const int c = (int)(rec[q].x & 0xffu);
        const float v = __uint_as_float(rec[q].y);
        const uint32_t eb = T.gs[g], ee = T.gs[g + 1];
        for (uint32_t e = eb; e < ee; ++e)
          atomicAdd(&acc[(int)T.er[e] * ld + c], tail_fixed(T.eu[e] * v));
      }
    }
  }
}

}  // namespace cuapss
