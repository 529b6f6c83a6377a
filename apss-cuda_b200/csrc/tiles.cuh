// Launch interfaces of the pair-tile kernels and the finalize stage.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"
#include "side.cuh"

namespace cuapss {

// Arguments shared by the pair-tile kernels. A unit of work is one I row
// block against a contiguous range [J0, J1) of J row blocks; the host cuts
// heavy I blocks into short J ranges so that units cost about the same, and
// the CTAs take units from a global counter.
struct TileArgs {
  // I side (rows of the tile)
  const float* headI32;
  const void* headI16;
  int64_t nI;
  int nbI;
  const int32_t* blkmaxI;
  const float* hnormI;
  const int64_t* bptrI;     // tail postings of each I block
  const uint32_t* bilI_key; // {bucket << 15 | tag << 7 | row}, (bucket, tag, row) order
  const float* bilI_u;
  const uint8_t* bilI_len;  // feature run length at its first posting
  int64_t max_tailI;        // largest I-block tail (postings): picks the staging variant
  // J side (columns of the tile)
  const float* headJ32;
  const void* headJ16;
  int64_t nJ;
  int nbJ;
  const int32_t* blkmaxJ;
  const float* hnormJ;
  const int64_t* hptrJ;     // postings of each kJSegRows-row segment of J
  const uint2* bilJ_rec;    // packed postings {feature << 8 | row, value bits}
  // explicit pairs of rare features (self-joins; null: none): records of
  // tile (I, J) at [ex_off[t], ex_off[t + 1]), t = tile_index(I, J, nbI):
  // {fixed-point product << 32 | row in I block << 7 | column in J block}
  const uint32_t* ex_off;
  const uint64_t* ex_rec;
  int p;
  int self;
  float t;
  const float* t_row;  // threshold of each I row (batched instances, queries), or null: t
  double eps_c1;  // FP32 error margin of a tile: eps_c1 * min(maxnnz_I, maxnnz_J) + eps_c0
  double eps_c0;
  double eps_head;  // tensor-core path: extra margin per unit of ||a_h|| ||b_h||
  const int4* units;  // {I, J0, J1, 0}
  int nunits;
  int* unit_counter;
  uint64_t* cand_key;
  float* cand_sim;
  unsigned long long* cand_count;
  int64_t cand_cap;
  int* err;
};

// Error margins of the tile decision for rows of norm <= sqrt(nrm2) and head
// width ta.p. FP32 head chain + fixed-point tail (2^-30 grid, exact sums) +
// final add: |s~ - s| <= (K + 3) u ||a|| ||b|| + K 2^-31, K = shared
// features. Tensor-core head (mixed): each BF16 factor is rounded to 8
// significant bits (relative 2^-8), products are exact in FP32, and the
// accumulation over p/16 MMA steps is bounded by 2^-20 relative per step.
inline void set_tile_margins(TileArgs& ta, double nrm2, bool mixed) {
  const double u = std::ldexp(1.0, -24);
  ta.eps_c1 = (u * nrm2 + std::ldexp(1.0, -31)) * 1.001;
  ta.eps_c0 = 3.0 * u * nrm2 * 1.001 + 1e-10;
  ta.eps_head = 0.0;
  if (mixed) {
    ta.eps_head = (std::ldexp(1.0, -7) + std::ldexp(1.0, -16)) +
                  (ta.p / 16.0 + 2.0) * std::ldexp(1.0, -20) * (1.0 + std::ldexp(1.0, -7));
    ta.eps_head *= 1.001;
  }
}

// Orders units so that the CTAs running at the same time share operands in
// L2: units are grouped by the window of J blocks they start in (window =
// the median J-range length) and ordered by I inside a group. The ~148
// concurrent units then read a few J blocks (L2 hits) against different I
// blocks, instead of one I block against 148 different J ranges.
inline void order_units_for_l2(std::vector<int4>& units) {
  if (units.size() < 2) return;
  std::vector<int> len(units.size());
  for (size_t k = 0; k < units.size(); ++k) len[k] = units[k].z - units[k].y;
  std::nth_element(len.begin(), len.begin() + len.size() / 2, len.end());
  const int w = std::max(1, len[len.size() / 2]);
  std::stable_sort(units.begin(), units.end(), [w](const int4& a, const int4& b) {
    const int wa = a.y / w, wb = b.y / w;
    return wa != wb ? wa < wb : a.x < b.x;
  });
}

// Plain FP32 hybrid tile kernel (head: FP32 forward-list dot on TMA-staged
// row tiles; tail: inverted-list scan into shared-memory accumulators).
// overlap_prev: the launch may start while the previous kernel on the
// stream still runs (programmatic dependent launch), taking the SMs its
// CTAs leave; only for work independent of that kernel's results.
cuapss_status launch_tiles_fp32(const TileArgs& a, int grid, cudaStream_t st,
                                bool overlap_prev = false);
cuapss_status tiles_fp32_init();
int tiles_fp32_max_grid();

// Mixed-precision tile kernel (BF16 head on tcgen05 tensor cores, FP32 tail).
// headI16 / headJ16: BF16 head blocks in the swizzled layout of
// build_side; p a multiple of 64. head_bound: the head's operand stream
// dominates the tiles (the caller's cost model puts the head at least twice
// the tail), so MMA tiles of two J blocks are used where the tail staging
// fits them.
cuapss_status launch_tiles_mma(const TileArgs& a, const void* headI16, const void* headJ16,
                               int p, int grid, cudaStream_t st, bool overlap_prev = false,
                               bool head_bound = false);
size_t tiles_mma_smem_bytes();
cuapss_status tiles_mma_init();

// Kernel attributes of the tile kernel of a precision, on the current device.
inline cuapss_status tiles_init(bool mixed) { return mixed ? tiles_mma_init() : tiles_fp32_init(); }

struct FinalizeArgs {
  const uint64_t* cand_key;
  const float* cand_sim;
  int64_t ncand;
  const int32_t* rowpermI;
  const int32_t* rowpermJ;
  const int32_t* nnzI;
  const int32_t* nnzJ;
  const float* hnormI;
  const float* hnormJ;
  const int64_t* rpI;
  const int32_t* colI;
  const float* valI;
  const int64_t* rpJ;
  const int32_t* colJ;
  const float* valJ;
  float t;
  const float* t_row;       // threshold of each I row, or null: t
  const int32_t* slot_row;  // side row -> caller's row (-1: padding), or null: rowperm
  int64_t j_offset;         // added to the J row of every output pair (index segments)
  double eps_c1;
  double eps_c0;
  double eps_head;
  int self;
  int rbits;  // output key = (i << rbits) | j
  uint64_t* out_key;
  uint32_t* out_idx;
  float* out_sim;
  unsigned long long* out_count;
  int64_t out_cap;
  unsigned long long* n_rescored;
};

cuapss_status launch_finalize(const FinalizeArgs& a, cudaStream_t st);

// After sorting out_key (with out_idx as payload): split into i, j, sim.
cuapss_status launch_split_pairs(const uint64_t* key, const uint32_t* idx, const float* sim_in,
                                 int64_t m, int rbits, int32_t* oi, int32_t* oj, float* os,
                                 cudaStream_t st);

}  // namespace cuapss
