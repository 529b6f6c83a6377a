// Device-resident layout of one operand of a similarity join, after
// validation, frequency remap and the index build.
//
// HBM layout (n rows, d features, nnz non-zeros, p head width, nb = ceil(n/128)
// row blocks of 128 rows, T tail non-zeros):
//   rowperm   int32[n]        row -> caller's row (rows keep the caller's
//                             order: the identity)
//   rp2       int64[n+1]      copy of the caller's rowptr
//   col2/val2 int32/f32[nnz]  the tail entries of each row (features of rank
//                             >= p, remapped to their frequency rank), as a
//                             suffix of the row's range (tptr counts them);
//                             for a self-join the rare features' entries as
//                             its prefix; the head entries are not written
//   head32    f32[nb][p][128] dense head block, k-major inside a row block so
//                             that a 32-feature slice of a block is one
//                             contiguous 16 KB run (one bulk TMA copy)
//   head16    bf16            dense head block for the tensor-core path
//   cptr/csc  int64[d-p+1], {int32 row, f32 val}[T]
//                             inverted lists of the tail features (rank >= p),
//                             rows ascending: the global index (built on
//                             request)
//   tptr      int64[n+1]      tail entries of each row, in row order
//   bptr      int64[nb+1]     tail entries of each row block
//   bil_key/bil_u/bil_len     block-local inverted lists: the tail postings
//                             of each row block sorted by (bucket = f mod
//                             2^12, tag = f >> 12, row), f = feature - p:
//                             key {bucket << 15 | tag << 7 | row in block},
//                             value, and the length of each feature's run at
//                             its first posting
//   bil_rec   uint2[T]        the same postings per kJSegRows-row segment,
//                             sorted by feature, packed {feature << 8 | row in
//                             block, value}
//   hptr      int64[kJSegs nb + 1]  postings of each J segment
#pragma once

#include <cuda_bf16.h>

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace cuapss {

struct Side {
  int64_t n = 0, d = 0, nnz = 0;
  int nb = 0;       // row blocks of kBlockRows
  int p = 0;        // head width
  // caller's CSR on the device (input pointers or a staged copy)
  const int64_t* rp0 = nullptr;
  const int32_t* col0 = nullptr;
  const float* val0 = nullptr;
  int32_t* rowperm = nullptr;
  int64_t* rp2 = nullptr;
  int32_t* col2 = nullptr;
  float* val2 = nullptr;
  int32_t* hlen = nullptr;
  int32_t* nnz_row = nullptr;
  int32_t* blk_maxnnz = nullptr;  // [nb]
  float* hnorm = nullptr;         // head norm (rounded up), new row order
  float* head32 = nullptr;
  __nv_bfloat16* head16 = nullptr;
  int64_t* tptr = nullptr;
  uint32_t* tk = nullptr;         // tail entry -> index into col2/val2
  int64_t* cptr = nullptr;
  uint2* csc = nullptr;
  uint8_t* tr = nullptr;          // row-order tail entries: row in block, value
  float* tu = nullptr;
  int64_t* bptr = nullptr;
  uint32_t* bil_key = nullptr;    // I-side postings {bucket << 15 | tag << 7 | row}
  float* bil_u = nullptr;
  uint8_t* bil_len = nullptr;     // run length at a feature's first posting, else 0
  uint2* bil_rec = nullptr;       // J-side postings per kJSegRows-row segment, sorted by
                                  // feature: {feature << 8 | row in block, value bits}
  int64_t* hptr = nullptr;        // [kJSegs nb + 1] postings of each J segment
  int64_t ntail = 0;
  int64_t max_block_tail = 0;
  std::vector<int64_t> h_bptr;    // host copy of bptr (unit scheduling)
  int64_t tail_products = 0;      // sum over tail lists of L(L-1)/2
  // explicit pairs of the rare features (self-joins): records grouped by
  // triangular tile index, {fixed-point product << 32 | row in I block << 7
  // | column in J block}; ex_off[t] = first record of tile t
  uint32_t* ex_off = nullptr;
  uint64_t* ex_rec = nullptr;
  int64_t n_explicit = 0;
  double nrm_max = 1.0;           // largest row norm (FP64)
};

}  // namespace cuapss
