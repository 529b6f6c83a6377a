// Tail phase shared by the pair-tile kernels: the sparse, feature-parallel
// part of the hybrid similarity.
//
// I side (the rows of a tile; fixed for a unit of work): the block-local
// inverted list of the 128-row block, grouped by feature, is staged in
// shared memory: the postings (row in block, value), the first posting of
// every group, and a hash of the group features. The hash is an array of
// 16-byte buckets of 4 packed slots {(feature + 1) << 12 | group}; a lookup
// reads one bucket (one 128-bit shared load) and compares four keys, and
// only a full bucket sends it to the next one. A block larger than the
// staging capacity (kGroupCap groups, ecap postings) is staged in chunks of
// consecutive groups, whose boundaries are computed once per block by the
// preprocessing.
//
// J side (the columns; one per tile): the tail postings of each 64-row
// half-block sorted by feature, packed as {feature << 8 | column, value}.
// Each posting (c, f, v) whose feature the I block contains adds u * v for
// every I posting (r, u) of that group into the shared-memory accumulator
// acc[r][c] with an integer atomic on a fixed-point grid of 2^-30: FP32
// products are rounded to the grid and the integer sums are exact in any
// order, so the tail is deterministic and its error is the product rounding
// plus 2^-31 per term.
//
// This replaces the reference's per-feature block schedule and its
// global-memory float atomics into a dense n x n array (fengyilin118/
// APSS-CUDA generate_auxiliary_variable{,2}{,_apss} and similarity_join1 /
// similarity_apss1, similarity_search.cu:323-437 and 577-735).
#pragma once

#include "ptx.cuh"
#include "tiles.cuh"

namespace cuapss {

constexpr int kGroupCap = kChunkGroups;  // groups per staged chunk (12-bit slot value)
static_assert(kGroupCap <= 4096, "slot value is 12 bits");
constexpr int kBuckets = 2048;        // hash buckets of 4 slots (load <= 1/2)
constexpr uint32_t kMaxTailFeature = (1u << 20) - 2;  // 20-bit slot key = feature + 1
constexpr float kTailScale = 1073741824.0f;              // 2^30
constexpr float kTailUnscale = 9.313225746154785e-10f;   // 2^-30

__device__ __forceinline__ int tail_fixed(float prod) { return __float2int_rn(prod * kTailScale); }

__device__ __forceinline__ uint32_t tail_bucket(uint32_t f) {
  return (f * 2654435761u) >> (32 - 11);  // 11 bits: kBuckets
}

// Shared-memory staging buffers of the I side.
struct TailStage {
  uint4* hash;     // [kBuckets] 4 packed slots each, 0 = empty
  uint16_t* gs;    // [kGroupCap + 1] first posting of each group (chunk relative)
  uint8_t* er;     // [ecap] posting: row in block
  float* eu;       // [ecap] posting: value
  int ecap;
};

// The staged chunk.
struct TailI {
  int G;
  bool any;
};

template <int NT, int BAR>
__device__ __forceinline__ void tail_sync() {
  if (BAR == 0) __syncthreads();
  else named_bar(BAR, NT);
}

// Chunks of I block I: chunk c holds the groups
// [chunk_gI[chunk_ptrI[I] + c], chunk_gI[chunk_ptrI[I] + c + 1]).
__device__ __forceinline__ int tail_nchunks(const TileArgs& A, int I) {
  return (int)(A.chunk_ptrI[I + 1] - A.chunk_ptrI[I]) - 1;
}

// Stage chunk c of block I. All NT tail threads (ltid = index among them)
// call it; it ends with a tail barrier.
template <int NT, int BAR>
__device__ __forceinline__ TailI stage_tail_chunk(const TileArgs& A, const TailStage& S, int I,
                                                  int c, int ltid) {
  const int64_t cb = A.chunk_ptrI[I] + c;
  const int64_t ga = A.chunk_gI[cb], gb = A.chunk_gI[cb + 1];
  const uint32_t e0 = A.gstartI[ga];
  const uint32_t e1 = A.gstartI[gb];
  TailI T;
  T.G = (int)(gb - ga);
  T.any = T.G > 0;
  for (int w = ltid; w < kBuckets; w += NT) S.hash[w] = make_uint4(0u, 0u, 0u, 0u);
  tail_sync<NT, BAR>();
  uint32_t* slots = reinterpret_cast<uint32_t*>(S.hash);
  for (int g = ltid; g < T.G; g += NT) {
    const uint32_t f = A.gfeatI[ga + g];
    S.gs[g] = (uint16_t)(A.gstartI[ga + g] - e0);
    const uint32_t key = ((f + 1u) << 12) | (uint32_t)g;
    uint32_t b = tail_bucket(f);
    for (int probe = 0; probe < kBuckets; ++probe) {
      bool done = false;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (atomicCAS(&slots[b * 4 + k], 0u, key) == 0u) {
          done = true;
          break;
        }
      }
      if (done) break;
      b = (b + 1u) & (kBuckets - 1);
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
__device__ __forceinline__ int find_group(const TailStage& S, uint32_t f) {
  const uint32_t want = f + 1u;
  uint32_t b = tail_bucket(f);
  for (int probe = 0; probe < kBuckets; ++probe) {
    const uint4 q = S.hash[b];
    if ((q.x >> 12) == want) return (int)(q.x & 0xfffu);
    if ((q.y >> 12) == want) return (int)(q.y & 0xfffu);
    if ((q.z >> 12) == want) return (int)(q.z & 0xfffu);
    if ((q.w >> 12) == want) return (int)(q.w & 0xfffu);
    if (q.w == 0u) return -1;  // a bucket fills in slot order: not full, not here
    b = (b + 1u) & (kBuckets - 1);
  }
  return -1;
}

// Products of one matched J posting (column c, value v) with group g.
__device__ __forceinline__ void tail_products(const TailStage& S, int g, int c, float v, int* acc,
                                              int ld) {
  const uint32_t eb = S.gs[g], ee = S.gs[g + 1];
  int* col = acc + c;
  uint32_t e = eb;
  for (; e + 1 < ee; e += 2) {
    const int r0 = S.er[e], r1 = S.er[e + 1];
    const float u0 = S.eu[e], u1 = S.eu[e + 1];
    atomicAdd(col + r0 * ld, tail_fixed(u0 * v));
    atomicAdd(col + r1 * ld, tail_fixed(u1 * v));
  }
  if (e < ee) atomicAdd(col + (int)S.er[e] * ld, tail_fixed(S.eu[e] * v));
}

// Tail contributions of the J postings [k0, k1) (column = record & 0xff,
// minus cofs) against the staged chunk, into acc[r * ld + c - cofs]; thread
// tid of nthreads; NB postings per thread are loaded before they are used.
template <int NB>
__device__ __forceinline__ void tail_postings(const TileArgs& A, const TailStage& S,
                                              const TailI& T, int64_t k0, int64_t k1, int* acc,
                                              int ld, int cofs, int tid, int nthreads) {
  if (!T.any) return;
  const int n = (int)(k1 - k0);
  for (int kb = tid; kb < n; kb += NB * nthreads) {
    uint2 rec[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int k = kb + q * nthreads;
      rec[q] = k < n ? __ldg(&A.bilJ_rec[k0 + k]) : make_uint2(0xffffffffu, 0u);
    }
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      if (rec[q].x == 0xffffffffu) break;  // the rest of the batch is past the range
      const int g = find_group(S, rec[q].x >> 8);
      if (g >= 0)
        tail_products(S, g, (int)(rec[q].x & 0xffu) - cofs, __uint_as_float(rec[q].y), acc, ld);
    }
  }
}

}  // namespace cuapss
