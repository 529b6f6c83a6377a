// Finalize stage: decides every candidate pair exactly and computes the
// similarity that is reported.
//
// A candidate left a tile with an approximate similarity s~ and a proven
// error bound eps (FP32 rounding, plus BF16 input rounding on the
// tensor-core path). With s64 the FP64 similarity of the oracle:
//   s~ - eps >= t  -> in; the reported value is a compensated FP32 dot
//                     (Ogita-Rump-Oishi Dot2: TwoProduct by FMA + TwoSum),
//                     within ~1.2e-7 of s64;
//   otherwise       -> rescored in FP64, accumulating in ascending feature
//                     order exactly as the oracle does, so the in/out decision
//                     is bit-identical to the oracle's.
// The reference has no such stage: its threshold test is an empty branch
// (fengyilin118/APSS-CUDA similarity_search.cu:498-502, 907-911).
#include <cuda_runtime.h>

#include "tiles.cuh"

namespace cuapss {

namespace {

constexpr int kThreads = 256;

// FP64 merge-dot over two rows sorted by feature id (oracle order).
__device__ double dot_fp64(const int32_t* __restrict__ ca, const float* __restrict__ va, int64_t na,
                           const int32_t* __restrict__ cb, const float* __restrict__ vb, int64_t nb) {
  double s = 0.0;
  int64_t a = 0, b = 0;
  while (a < na && b < nb) {
    const int32_t x = ca[a], y = cb[b];
    if (x < y) {
      ++a;
    } else if (x > y) {
      ++b;
    } else {
      s = __dadd_rn(s, __dmul_rn((double)va[a], (double)vb[b]));
      ++a;
      ++b;
    }
  }
  return s;
}

// Compensated FP32 merge-dot (Dot2).
__device__ float dot2_fp32(const int32_t* __restrict__ ca, const float* __restrict__ va, int64_t na,
                           const int32_t* __restrict__ cb, const float* __restrict__ vb, int64_t nb) {
  float s = 0.0f, c = 0.0f;
  int64_t a = 0, b = 0;
  while (a < na && b < nb) {
    const int32_t x = ca[a], y = cb[b];
    if (x < y) {
      ++a;
    } else if (x > y) {
      ++b;
    } else {
      const float u = va[a], v = vb[b];
      const float p = __fmul_rn(u, v);
      const float q = __fmaf_rn(u, v, -p);           // TwoProduct error
      const float sn = __fadd_rn(s, p);              // TwoSum
      const float z = __fsub_rn(sn, s);
      const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(sn, z)), __fsub_rn(p, z));
      s = sn;
      c = __fadd_rn(c, __fadd_rn(e, q));
      ++a;
      ++b;
    }
  }
  return __fadd_rn(s, c);
}

__global__ void __launch_bounds__(kThreads) k_finalize(const FinalizeArgs A) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < A.ncand;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = A.cand_key[q];
    const int32_t inew = (int32_t)(key >> 32), jnew = (int32_t)(key & 0xffffffffu);
    const float st = A.cand_sim[q];
    const int K = min(A.nnzI[inew], A.nnzJ[jnew]);
    double eps = A.eps_c1 * K + A.eps_c0;
    if (A.eps_head > 0.0) eps += A.eps_head * (double)A.hnormI[inew] * (double)A.hnormJ[jnew];
    const double lo = (double)st - eps, hi = (double)st + eps;
    const double t = A.t_row ? (double)A.t_row[inew] : (double)A.t;
    if (hi < t) continue;
    const int32_t oi = A.rowpermI[inew], oj = A.rowpermJ[jnew];
    const int64_t ai = A.rpI[oi], an = A.rpI[oi + 1] - ai;
    const int64_t bj = A.rpJ[oj], bn = A.rpJ[oj + 1] - bj;
    float sim;
    bool in;
    if (lo >= t) {
      in = true;
      sim = dot2_fp32(A.colI + ai, A.valI + ai, an, A.colJ + bj, A.valJ + bj, bn);
    } else {
      atomicAdd(A.n_rescored, 1ull);
      // FP64 in the oracle's order: the self-join oracle walks the lower id's
      // row, which for a product of two exact factors gives the same sums.
      const double s64 = dot_fp64(A.colI + ai, A.valI + ai, an, A.colJ + bj, A.valJ + bj, bn);
      in = s64 >= t;
      sim = (float)s64;
    }
    if (!in) continue;
    int32_t ri = oi, rj = oj;
    if (A.slot_row) {
      ri = A.slot_row[oi];
      rj = A.slot_row[oj];
      if (ri < 0 || rj < 0) continue;  // padding rows (empty) of a batched layout
    }
    uint64_t a = (uint64_t)ri, b = (uint64_t)((int64_t)rj + A.j_offset);
    if (A.self && a > b) {
      const uint64_t tmp = a;
      a = b;
      b = tmp;
    }
    const unsigned long long w = atomicAdd(A.out_count, 1ull);
    if ((int64_t)w < A.out_cap) {
      A.out_key[w] = (a << A.rbits) | b;
      A.out_idx[w] = (uint32_t)w;
      A.out_sim[w] = sim;
    }
  }
}

__global__ void k_split_pairs(const uint64_t* __restrict__ key, const uint32_t* __restrict__ idx,
                              const float* __restrict__ sim_in, int64_t m, int rbits,
                              int32_t* __restrict__ oi, int32_t* __restrict__ oj,
                              float* __restrict__ os) {
  const uint64_t mask = (1ull << rbits) - 1ull;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = key[q];
    oi[q] = (int32_t)(k >> rbits);
    oj[q] = (int32_t)(k & mask);
    os[q] = sim_in[idx[q]];
  }
}

}  // namespace

cuapss_status launch_finalize(const FinalizeArgs& a, cudaStream_t st) {
  if (a.ncand <= 0) return CUAPSS_OK;
  const int64_t g = std::min<int64_t>(ceil_div(a.ncand, kThreads), 148 * 16);
  k_finalize<<<(unsigned)g, kThreads, 0, st>>>(a);
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

cuapss_status launch_split_pairs(const uint64_t* key, const uint32_t* idx, const float* sim_in,
                                 int64_t m, int rbits, int32_t* oi, int32_t* oj, float* os,
                                 cudaStream_t st) {
  if (m <= 0) return CUAPSS_OK;
  const int64_t g = std::min<int64_t>(ceil_div(m, kThreads), 148 * 16);
  k_split_pairs<<<(unsigned)g, kThreads, 0, st>>>(key, idx, sim_in, m, rbits, oi, oj, os);
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

}  // namespace cuapss
