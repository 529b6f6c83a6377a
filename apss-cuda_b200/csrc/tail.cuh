// Tail phase shared by the pair-tile kernels: the sparse, feature-parallel
// part of the hybrid similarity.
//
// I side (the rows of a tile; fixed for a unit of work): the block-local
// inverted list of the 128-row block is staged in shared memory as a
// bucketed posting list. The preprocessing sorts the block's tail postings
// by (bucket = f mod 2^12, tag = f >> 12, row), f the tail feature, so a
// staged posting is {tag << 7 | row} (16 bits), its value (FP32) and, at the
// first posting of each feature's run, the run length (8 bits); a table of
// 4097 bucket offsets (16 bits each) delimits the buckets. Staging is a
// straight copy plus the offsets: no hashing, no atomics. A block with more
// postings than the staging capacity is staged in consecutive chunks of that
// many postings (any cut is valid: every chunk adds the products
// of its own postings; a run cut by a chunk boundary is re-measured).
//
// J side (the columns; one per tile): the tail postings of each
// kJSegRows-row segment of the J block sorted by feature, packed as
// {feature << 8 | column, value}.
// A J posting (c, f, v) reads the two offsets of bucket f mod 2^12 and walks
// that bucket run by run (tags ascend) to the run with tag f >> 12; each of
// its postings (r, u) adds u * v into the shared-memory accumulator
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

constexpr int kStagePostings = 12800;  // default postings per staged chunk (16-bit offsets)
constexpr uint32_t kMaxTailFeature = (1u << 20) - 1;  // 8-bit tag above 12-bit bucket
constexpr float kTailScale = 1073741824.0f;              // 2^30
constexpr float kTailUnscale = 9.313225746154785e-10f;   // 2^-30

constexpr size_t kTailOffBytes = ((size_t)(kTailBuckets + 1) * 2 + 15) / 16 * 16;
// Shared memory of CAP staged I postings.
template <int CAP>
constexpr size_t tail_stage_bytes() {
  static_assert(CAP > 0 && CAP < 65536 && CAP % 16 == 0, "bucket offsets are 16 bits");
  return kTailOffBytes + (size_t)CAP * 7;
}
constexpr size_t kTailStageBytes = tail_stage_bytes<kStagePostings>();

__device__ __forceinline__ int tail_fixed(float prod) { return __float2int_rn(prod * kTailScale); }

// Shared-memory staging buffers of the I side.
struct TailStage {
  uint16_t* boff;  // [kTailBuckets + 1] first posting of each bucket
  float* eu;       // [CAP] posting: value
  uint16_t* et;    // [CAP] posting: tag << 7 | row in block
  uint8_t* en;     // [CAP] run length at a run's first posting
};

// Carves a TailStage of CAP postings out of tail_stage_bytes<CAP>() bytes of
// 16-byte aligned shared memory.
template <int CAP = kStagePostings>
__device__ __forceinline__ TailStage tail_stage_at(uint8_t* base) {
  TailStage t;
  t.boff = reinterpret_cast<uint16_t*>(base);
  t.eu = reinterpret_cast<float*>(base + kTailOffBytes);
  t.et = reinterpret_cast<uint16_t*>(base + kTailOffBytes + (size_t)CAP * 4);
  t.en = base + kTailOffBytes + (size_t)CAP * 6;
  return t;
}

// The staged chunk.
struct TailI {
  int P;     // postings staged
  bool any;
};

template <int NT, int BAR>
__device__ __forceinline__ void tail_sync() {
  if (BAR == 0) __syncthreads();
  else named_bar(BAR, NT);
}

// Chunks of CAP postings of I block I (at least one, possibly empty).
template <int CAP = kStagePostings>
__device__ __forceinline__ int tail_nchunks(const TileArgs& A, int I) {
  const int64_t T = A.bptrI[I + 1] - A.bptrI[I];
  return T <= CAP ? 1 : (int)((T + CAP - 1) / CAP);
}

// Stage chunk c of block I. All NT tail threads (ltid = index among them)
// call it; it ends with a tail barrier.
template <int NT, int BAR, int CAP = kStagePostings>
__device__ __forceinline__ TailI stage_tail_chunk(const TileArgs& A, const TailStage& S, int I,
                                                  int c, int ltid) {
  const int64_t b1 = A.bptrI[I + 1];
  const int64_t e0 = A.bptrI[I] + (int64_t)c * CAP;
  const int64_t rem = b1 - e0;
  const int P = rem <= 0 ? 0 : (rem < CAP ? (int)rem : CAP);
  TailI T;
  T.P = P;
  T.any = P > 0;
  if (P == 0) {
    for (int b = ltid; b <= (int)kTailBuckets; b += NT) S.boff[b] = 0;
  }
  for (int e = ltid; e < P; e += NT) {
    const uint32_t key = __ldg(&A.bilI_key[e0 + e]);
    S.et[e] = (uint16_t)(key & 0x7fffu);
    S.eu[e] = __ldg(&A.bilI_u[e0 + e]);
    int len = __ldg(&A.bilI_len[e0 + e]);
    if (e == 0 && len == 0) {
      // the chunk starts inside a run: measure what is left of it
      const uint32_t fk = key >> 7;
      len = 1;
      while (len < P && len < kBlockRows && (__ldg(&A.bilI_key[e0 + len]) >> 7) == fk) ++len;
    }
    S.en[e] = (uint8_t)(len < P - e ? len : P - e);
    // offsets: this posting starts every bucket after its predecessor's
    const int bk = (int)(key >> 15);
    const int bp = e > 0 ? (int)(__ldg(&A.bilI_key[e0 + e - 1]) >> 15) : -1;
    for (int b = bp + 1; b <= bk; ++b) S.boff[b] = (uint16_t)e;
    if (e == P - 1)
      for (int b = bk + 1; b <= (int)kTailBuckets; ++b) S.boff[b] = (uint16_t)P;
  }
  tail_sync<NT, BAR>();
  return T;
}

// Accumulator cell of (row r, column c): plain rows of ld ints, or (SWZ)
// rows of 32 ints whose 4-int groups are permuted by the row (group g of row
// r at position g ^ (r % 8)), so that eight consecutive rows' same group sit
// in distinct banks for the epilogue's 16-byte reads.
template <bool SWZ>
__device__ __forceinline__ int acc_cell(int r, int c, int ld) {
  return SWZ ? r * 32 + ((((c >> 2) ^ (r & 7)) << 2) | (c & 3)) : r * ld + c;
}

// Triangular index of tile (I, J), J >= I, among nb row blocks.
__host__ __device__ __forceinline__ int64_t tile_index(int64_t I, int64_t J, int64_t nb) {
  return I * nb - I * (I - 1) / 2 + (J - I);
}

// Adds the explicit rare-feature records [lo, hi) of a tile whose column
// lies in [cofs, cofs + ncols) into acc at acc_cell<SWZ>(row, column - cofs);
// thread tid of nthreads.
template <bool SWZ>
__device__ __forceinline__ void tail_explicit(const TileArgs& A, uint32_t lo, uint32_t hi,
                                              int* acc, int ld, int cofs, int ncols, int tid,
                                              int nthreads) {
  for (uint32_t k = lo + (uint32_t)tid; k < hi; k += (uint32_t)nthreads) {
    const uint64_t rec = __ldg(&A.ex_rec[k]);
    const int c = (int)(rec & 127u) - cofs;
    if (c >= 0 && c < ncols)
      atomicAdd(acc + acc_cell<SWZ>((int)((rec >> 7) & 127u), c, ld), (int)(rec >> 32));
  }
}

// Products of one J posting (feature f, column c, value v) with the staged
// I postings of feature f.
template <bool SWZ>
__device__ __forceinline__ void tail_probe(const TailStage& S, uint32_t f, int c, float v,
                                           int* acc, int ld) {
  const uint32_t b = f & (kTailBuckets - 1u);
  const uint32_t tag = f >> kTailBucketBits;
  int e = S.boff[b];
  const int e1 = S.boff[b + 1];
  while (e < e1) {
    const uint32_t tg = (uint32_t)S.et[e] >> 7;
    const int len = S.en[e];
    if (tg < tag) {
      e += len > 0 ? len : 1;  // next run of the bucket (every run start has len >= 1)
      continue;
    }
    if (tg == tag) {
      const int ee = e + len;
      for (; e + 1 < ee; e += 2) {
        const uint32_t t0 = S.et[e], t1 = S.et[e + 1];
        const float u0 = S.eu[e], u1 = S.eu[e + 1];
        atomicAdd(acc + acc_cell<SWZ>((int)(t0 & 127u), c, ld), tail_fixed(u0 * v));
        atomicAdd(acc + acc_cell<SWZ>((int)(t1 & 127u), c, ld), tail_fixed(u1 * v));
      }
      if (e < ee) atomicAdd(acc + acc_cell<SWZ>((int)(S.et[e] & 127u), c, ld), tail_fixed(S.eu[e] * v));
    }
    break;
  }
}

// Tail contributions of the J postings [k0, k1) (column = record & 0xff,
// minus cofs) against the staged chunk, into acc at acc_cell<SWZ>(r, c - cofs);
// thread tid of nthreads; NB postings per thread are loaded before they are
// used.
template <int NB, bool SWZ = false>
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
      tail_probe<SWZ>(S, rec[q].x >> 8, (int)(rec[q].x & 0xffu) - cofs,
                      __uint_as_float(rec[q].y), acc, ld);
    }
  }
}

}  // namespace cuapss
