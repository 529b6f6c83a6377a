// Tail phase shared by the pair-tile kernels: the sparse, feature-parallel
// part of the hybrid similarity.
//
// I side (the rows of a tile; fixed for a unit of work): the block-local
// inverted list of the 128-row block, grouped by feature (sorted feature,
// first posting) with postings (row in block, value), is staged in shared
// memory. A block whose list exceeds the staging capacity is staged in
// chunks of consecutive groups. A direct table maps the kWarm most frequent
// tail features to their group; a bloom bitmap rejects the other features
// that the block does not contain before a binary search over the groups.
//
// J side (the columns; one per tile): the tail postings of each 64-row
// half-block sorted by feature, packed as {feature << 8 | column, value},
// read with batched coalesced loads. Each posting (c, f, v) whose feature
// the I block contains adds u * v for every I posting (r, u) of that group
// into the shared-memory accumulator acc[r][c] with an integer atomic on a
// fixed-point grid of 2^-30: FP32 products are rounded to the grid and the
// integer sums are exact in any order, so the tail is deterministic and its
// error is the product rounding plus 2^-31 per term.
//
// This replaces the reference's per-feature block schedule and its
// global-memory float atomics into a dense n x n array (fengyilin118/
// APSS-CUDA generate_auxiliary_variable{,2}{,_apss} and similarity_join1 /
// similarity_apss1, similarity_search.cu:323-437 and 577-735).
#pragma once

#include "ptx.cuh"
#include "tiles.cuh"

namespace cuapss {

constexpr int kWarm = 4096;           // tail features with a direct table
constexpr int kBloomWords = 1024;     // 32768-bit filter for the other features
constexpr uint16_t kNoGroup = 0xffff;
constexpr float kTailScale = 1073741824.0f;              // 2^30
constexpr float kTailUnscale = 9.313225746154785e-10f;   // 2^-30

__device__ __forceinline__ int tail_fixed(float prod) { return __float2int_rn(prod * kTailScale); }

__device__ __forceinline__ uint32_t bloom_bit(uint32_t f) { return (f * 2654435761u) >> 17; }

// Shared-memory staging buffers of the I side (capacity `ecap` postings,
// at most `ecap` groups since every group holds at least one posting).
struct TailStage {
  uint32_t* gf;    // [ecap] feature of each group, ascending
  uint16_t* gs;    // [ecap + 1] first posting of each group (chunk relative)
  uint8_t* er;     // [ecap] posting: row in block
  float* eu;       // [ecap] posting: value
  uint16_t* warm;  // [kWarm] group of warm feature f, or kNoGroup
  uint32_t* bloom; // [kBloomWords]
  int ecap;
};

// The staged chunk.
struct TailI {
  int G;        // groups staged
  int gw;       // groups with a warm feature (a prefix)
  uint32_t flo, fhi;  // feature range of the chunk
  bool any;
};

// Chunking of an I block: chunk c holds the groups starting at the first
// group whose first posting is >= e0 + c * step, step = ecap - 128 (a group
// has at most 128 postings, so a chunk never exceeds ecap postings).
__device__ __forceinline__ int tail_nchunks(const TileArgs& A, int I, int ecap) {
  const int64_t g0 = A.gptrI[I], g1 = A.gptrI[I + 1];
  const int64_t e = (int64_t)A.gstartI[g1] - A.gstartI[g0];
  const int64_t step = ecap - 128;
  return e <= ecap ? 1 : (int)((e + step - 1) / step);
}

__device__ __forceinline__ int64_t tail_chunk_start(const TileArgs& A, int I, int c, int nch,
                                                    int ecap) {
  const int64_t g0 = A.gptrI[I], g1 = A.gptrI[I + 1];
  if (c <= 0) return g0;
  if (c >= nch) return g1;
  const uint32_t target = A.gstartI[g0] + (uint32_t)((int64_t)c * (ecap - 128));
  int64_t lo = g0, hi = g1;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (A.gstartI[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

template <int NT, int BAR>
__device__ __forceinline__ void tail_sync() {
  if (BAR == 0) __syncthreads();
  else named_bar(BAR, NT);
}

// Stage chunk c of block I. All NT tail threads (ltid = index among them)
// call it; it ends with a tail barrier.
template <int NT, int BAR>
__device__ __forceinline__ TailI stage_tail_chunk(const TileArgs& A, const TailStage& S, int I,
                                                  int c, int nch, int ltid) {
  const int64_t ga = tail_chunk_start(A, I, c, nch, S.ecap);
  const int64_t gb = tail_chunk_start(A, I, c + 1, nch, S.ecap);
  const uint32_t e0 = A.gstartI[ga];
  const uint32_t e1 = A.gstartI[gb];
  TailI T;
  T.G = (int)(gb - ga);
  T.any = T.G > 0;
  T.flo = T.any ? A.gfeatI[ga] : 0xffffffffu;
  T.fhi = T.any ? A.gfeatI[gb - 1] : 0u;
  for (int w = ltid; w < kWarm; w += NT) S.warm[w] = kNoGroup;
  for (int w = ltid; w < kBloomWords; w += NT) S.bloom[w] = 0u;
  {
    int lo = 0, hi = T.G;  // groups are sorted by feature: the warm ones form a prefix
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (A.gfeatI[ga + mid] < (uint32_t)kWarm) lo = mid + 1;
      else hi = mid;
    }
    T.gw = lo;
  }
  tail_sync<NT, BAR>();
  for (int g = ltid; g < T.G; g += NT) {
    const uint32_t f = A.gfeatI[ga + g];
    S.gf[g] = f;
    S.gs[g] = (uint16_t)(A.gstartI[ga + g] - e0);
    if (g < T.gw) {
      S.warm[f] = (uint16_t)g;
    } else {
      const uint32_t bit = bloom_bit(f);
      atomicOr(&S.bloom[bit >> 5], 1u << (bit & 31));
    }
  }
  if (ltid == 0) S.gs[T.G] = (uint16_t)(e1 - e0);
  for (uint32_t e = ltid; e < e1 - e0; e += NT) {
    S.er[e] = A.bilI_r[e0 + e];
    S.eu[e] = A.bilI_u[e0 + e];
  }
  tail_sync<NT, BAR>();
  return T;
}

// Group of feature f in the staged chunk, or -1.
__device__ __forceinline__ int find_group(const TailStage& S, const TailI& T, uint32_t f) {
  if (f < (uint32_t)kWarm) {
    const uint16_t g = S.warm[f];
    return g == kNoGroup ? -1 : (int)g;
  }
  const uint32_t bit = bloom_bit(f);
  if (!((S.bloom[bit >> 5] >> (bit & 31)) & 1u)) return -1;
  int lo = T.gw, hi = T.G;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (S.gf[mid] < f) lo = mid + 1;
    else hi = mid;
  }
  return (lo < T.G && S.gf[lo] == f) ? lo : -1;
}

// Matches a batch of J postings against the staged chunk and adds the
// products. Lookups are issued for the whole batch first (table or bloom
// word, predicated loads, no branches), then the rare binary searches, then
// the products for the hits.
template <int NB>
__device__ __forceinline__ void tail_match(const TileArgs& A, const TailStage& S, const TailI& T,
                                           const uint2 (&rec)[NB], int* acc, int ld, int cofs) {
  int g[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const uint32_t x = rec[q].x;
    const uint32_t f = x >> 8;
    const bool valid = x != 0xffffffffu && f >= T.flo && f <= T.fhi;
    const bool warm = f < (uint32_t)kWarm;
    const uint32_t bit = bloom_bit(f);
    const uint16_t w = (valid && warm) ? S.warm[f] : kNoGroup;
    const uint32_t bw = (valid && !warm) ? S.bloom[bit >> 5] : 0u;
    g[q] = warm ? (w == kNoGroup ? -1 : (int)w) : (((bw >> (bit & 31)) & 1u) ? -2 : -1);
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    if (g[q] == -2) {
      const uint32_t f = rec[q].x >> 8;
      int lo = T.gw, hi = T.G;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (S.gf[mid] < f) lo = mid + 1;
        else hi = mid;
      }
      g[q] = (lo < T.G && S.gf[lo] == f) ? lo : -1;
    }
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    if (g[q] >= 0) {
      const int c = (int)(rec[q].x & 0xffu) - cofs;
      const float v = __uint_as_float(rec[q].y);
      const uint32_t eb = S.gs[g[q]], ee = S.gs[g[q] + 1];
      int* col = acc + c;
      for (uint32_t e = eb; e < ee; ++e)
        atomicAdd(col + (int)S.er[e] * ld, tail_fixed(S.eu[e] * v));
    }
  }
}

// Tail contributions of the J postings [k0, k1) (one or two half-blocks of
// tile J's columns, column = record & 0xff, minus cofs) against the staged
// chunk, into acc[r * ld + c - cofs]; thread tid of nthreads.
template <int NB>
__device__ __forceinline__ void tail_postings(const TileArgs& A, const TailStage& S,
                                              const TailI& T, int64_t k0, int64_t k1, int* acc,
                                              int ld, int cofs, int tid, int nthreads) {
  if (!T.any) return;
  for (int64_t kb = k0 + tid; kb < k1; kb += (int64_t)NB * nthreads) {
    uint2 rec[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int64_t k = kb + (int64_t)q * nthreads;
      rec[q] = k < k1 ? __ldg(&A.bilJ_rec[k]) : make_uint2(0xffffffffu, 0u);
    }
    tail_match<NB>(A, S, T, rec, acc, ld, cofs);
  }
}

// Prefetched first batch of a J posting range: thread tid holds records
// k0 + tid + q * nthreads, q < NB.
template <int NB>
struct TailBatch {
  uint2 rec[NB];
  int64_t k0, k1;
};

template <int NB>
__device__ __forceinline__ void tail_prefetch(const TileArgs& A, TailBatch<NB>& B, int64_t k0,
                                              int64_t k1, int tid, int nthreads) {
  B.k0 = k0;
  B.k1 = k1;
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int64_t k = k0 + tid + (int64_t)q * nthreads;
    B.rec[q] = k < k1 ? __ldg(&A.bilJ_rec[k]) : make_uint2(0xffffffffu, 0u);
  }
}

// tail_postings with the first batch already loaded in B.
template <int NB>
__device__ __forceinline__ void tail_postings_pre(const TileArgs& A, const TailStage& S,
                                                  const TailI& T, const TailBatch<NB>& B, int* acc,
                                                  int ld, int cofs, int tid, int nthreads) {
  if (!T.any) return;
  tail_match<NB>(A, S, T, B.rec, acc, ld, cofs);
  const int64_t rest = B.k0 + (int64_t)NB * nthreads;
  if (rest < B.k1) tail_postings<NB>(A, S, T, rest, B.k1, acc, ld, cofs, tid, nthreads);
}

}  // namespace cuapss
