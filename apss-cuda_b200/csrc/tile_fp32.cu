// Plain FP32 hybrid pair-tile kernel.
//
// One CTA evaluates 128 x 128 pair tiles (I block of rows x J block of
// columns) of the similarity matrix:
//  1. tail, feature-parallel (tail.cuh): the J block's block-local inverted
//     list is merged against the I block's feature groups (staged in shared
//     memory) and every common feature adds u * v into a shared-memory
//     accumulator acc[r][c] with shared-memory atomics (the role of similarity_apss1 /
//     similarity_join1, fengyilin118/APSS-CUDA similarity_search.cu:370-437
//     and 642-735, which instead add into a dense n x n global array);
//  2. head, pair-parallel: the dense head blocks of I and J (p features, 32
//     at a time, one 16 KB bulk-TMA copy per operand and slice, double
//     buffered) are multiplied with an FP32 FMA chain, 8 x 8 pairs per
//     thread (the role of similarity_apss_rest / similarity_join_rest,
//     similarity_search.cu:441-506 and 854-915, which do a sparse-dense dot
//     per pair against a dense copy of the query's head);
//  3. epilogue: head + tail is compared with t - eps (eps bounds the FP32
//     rounding of the tile, so no pair with FP64 similarity >= t is lost;
//     the reference's prune filter_pair, 510-531, uses "<= t" and drops
//     pairs at exactly t); surviving pairs are compacted with a warp ballot
//     and one atomic per warp into the candidate list (the reference counts
//     nothing: its atomicAdd(sum_pair) is commented out, 501 and 910).
// Units of work (I block x range of J blocks) are taken from a global
// counter by persistent CTAs.
#include <cuda_runtime.h>

#include <mutex>

#include <climits>

#include "ptx.cuh"
#include "tail.cuh"
#include "tiles.cuh"

namespace cuapss {

namespace {

constexpr int kThreads = 256;
constexpr int kKC = 32;                           // head features per slice
constexpr int kSlice = kKC * kBlockRows;          // floats per slice (4096)
constexpr int kSliceBytes = kSlice * 4;           // 16 KB
constexpr int kAccLd = kBlockRows + 4;            // padded accumulator row
constexpr size_t kOffAcc = 4 * (size_t)kSliceBytes;
constexpr size_t kOffBar = kOffAcc + (size_t)kBlockRows * kAccLd * 4;
constexpr size_t kOffTail = kOffBar + 64;                       // 16-byte aligned
constexpr size_t kSmemBytes = kOffTail + kTailStageBytes;
static_assert(kSmemBytes + 256 <= 232448, "shared memory budget");

struct Smem {
  float* a[2];
  float* b[2];
  float* acc;
  uint64_t* bar;
  TailStage ts;
};

__device__ __forceinline__ Smem carve(unsigned char* base) {
  Smem s;
  s.a[0] = reinterpret_cast<float*>(base);
  s.a[1] = s.a[0] + kSlice;
  s.b[0] = s.a[1] + kSlice;
  s.b[1] = s.b[0] + kSlice;
  s.acc = reinterpret_cast<float*>(base + kOffAcc);
  s.bar = reinterpret_cast<uint64_t*>(base + kOffBar);
  s.ts = tail_stage_at(base + kOffTail);
  return s;
}

__device__ __forceinline__ void issue_slice(const Smem& s, int stage, const float* headI,
                                            const float* headJ, int I, int J, int p, int kc) {
  mbar_arrive_expect_tx(&s.bar[stage], 2 * kSliceBytes);
  bulk_g2s(s.a[stage], headI + ((int64_t)I * p + (int64_t)kc * kKC) * kBlockRows, kSliceBytes,
           &s.bar[stage]);
  bulk_g2s(s.b[stage], headJ + ((int64_t)J * p + (int64_t)kc * kKC) * kBlockRows, kSliceBytes,
           &s.bar[stage]);
}

__global__ void __launch_bounds__(kThreads, 1) k_tiles_fp32(const TileArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const Smem S = carve(smem_raw);
  __shared__ int s_unit;
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int lane = tid & 31;
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    fence_mbar_init();
  }
  for (int i = tid; i < kBlockRows * kAccLd; i += kThreads) reinterpret_cast<int*>(S.acc)[i] = 0;
  __syncthreads();
  allow_dependent_launch();
  uint32_t parity[2] = {0u, 0u};
  const int nchunks = A.p / kKC;

  for (;;) {
    if (tid == 0) s_unit = atomicAdd(A.unit_counter, 1);
    __syncthreads();
    const int u = s_unit;
    __syncthreads();
    if (u >= A.nunits) break;
    const int4 U = A.units[u];
    if (U.y >= U.z) continue;
    const int I = U.x;
    const int64_t row0 = (int64_t)I * kBlockRows;
    const int rowsI = (int)(A.nI - row0 < kBlockRows ? A.nI - row0 : kBlockRows);
    const int nch = tail_nchunks(A, I);
    TailI T{};
    if (nch == 1) T = stage_tail_chunk<kThreads, 0>(A, S.ts, I, 0, tid);
    {
      for (int J = U.y; J < U.z; ++J) {
        const int64_t col0 = (int64_t)J * kBlockRows;
        if (tid == 0 && nchunks > 0) issue_slice(S, 0, A.headI32, A.headJ32, I, J, A.p, 0);
        // ---- tail: J's postings probe I's staged feature groups
        {
          int* acc = reinterpret_cast<int*>(S.acc);
          const int64_t k0 = A.hptrJ[kJSegs * J], k1 = A.hptrJ[kJSegs * (J + 1)];
          if (nch == 1) {
            tail_postings<8>(A, S.ts, T, k0, k1, acc, kAccLd, 0, tid, kThreads);
          } else {
            for (int c = 0; c < nch; ++c) {
              const TailI Tc = stage_tail_chunk<kThreads, 0>(A, S.ts, I, c, tid);
              tail_postings<8>(A, S.ts, Tc, k0, k1, acc, kAccLd, 0, tid, kThreads);
              __syncthreads();  // staging rewritten by the next chunk
            }
          }
          if (A.ex_off) {  // explicit pairs of the rare features
            const int64_t te = tile_index(I, J, A.nbI);
            tail_explicit<false>(A, A.ex_off[te], A.ex_off[te + 1], acc, kAccLd, 0, kBlockRows,
                                 tid, kThreads);
          }
        }
        // ---- head: FP32 FMA chain over the p head features
        float h[8][8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) h[i][j] = 0.0f;
        for (int kc = 0; kc < nchunks; ++kc) {
          const int stage = kc & 1;
          if (tid == 0 && kc + 1 < nchunks)
            issue_slice(S, stage ^ 1, A.headI32, A.headJ32, I, J, A.p, kc + 1);
          const bool ok = mbar_wait(&S.bar[stage], parity[stage]);
          parity[stage] ^= 1u;
          if (__syncthreads_or(!ok)) {
            if (tid == 0) {
              atomicOr(A.err, kErrTimeout);
              // the next slice's copy is in flight into the other stage: let
              // it land (bounded) before the CTA's shared memory goes away
              if (kc + 1 < nchunks) mbar_wait(&S.bar[stage ^ 1], parity[stage ^ 1]);
            }
            __syncthreads();
            return;
          }
          const float4* a4 = reinterpret_cast<const float4*>(S.a[stage]);
          const float4* b4 = reinterpret_cast<const float4*>(S.b[stage]);
#pragma unroll 8
          for (int k = 0; k < kKC; ++k) {
            const float4 a0 = a4[k * 32 + ty], a1 = a4[k * 32 + 16 + ty];
            const float4 b0 = b4[k * 32 + tx], b1 = b4[k * 32 + 16 + tx];
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
              for (int j = 0; j < 8; ++j) h[i][j] = fmaf(av[i], bv[j], h[i][j]);
          }
          __syncthreads();
        }
        if (nchunks == 0) __syncthreads();
        // ---- epilogue: head + tail >= t - eps  ->  candidates
        const int colsJ = (int)(A.nJ - col0 < kBlockRows ? A.nJ - col0 : kBlockRows);
        const bool diag = A.self && (I == J);
        const int kmax = min(A.blkmaxI[I], A.blkmaxJ[J]);
        const double margin = A.eps_c1 * kmax + A.eps_c0;
        float t_lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int r = (i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4);
          const double tr =
              A.t_row ? (r < rowsI ? (double)A.t_row[row0 + r] : 2.0) : (double)A.t;
          t_lo[i] = __double2float_rd(tr - margin);
        }
        unsigned long long pass = 0ull;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int r = (i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4);
          int4* arow = reinterpret_cast<int4*>(S.acc + r * kAccLd);
          const int4 t0 = arow[tx], t1 = arow[16 + tx];
          arow[tx] = make_int4(0, 0, 0, 0);
          arow[16 + tx] = make_int4(0, 0, 0, 0);
          const float tv[8] = {
              __int2float_rn(t0.x) * kTailUnscale, __int2float_rn(t0.y) * kTailUnscale,
              __int2float_rn(t0.z) * kTailUnscale, __int2float_rn(t0.w) * kTailUnscale,
              __int2float_rn(t1.x) * kTailUnscale, __int2float_rn(t1.y) * kTailUnscale,
              __int2float_rn(t1.z) * kTailUnscale, __int2float_rn(t1.w) * kTailUnscale};
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int c = (j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4);
            const float s = h[i][j] + tv[j];
            h[i][j] = s;
            const bool ok = (s >= t_lo[i]) && (r < rowsI) && (c < colsJ) && (!diag || c > r);
            pass |= (unsigned long long)ok << (i * 8 + j);
          }
        }
        if (__any_sync(0xffffffffu, pass != 0ull)) {
          const int mine = __popcll(pass);
          int incl = mine;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
          }
          const int total = __shfl_sync(0xffffffffu, incl, 31);
          unsigned long long base = 0;
          if (lane == 31) base = atomicAdd(A.cand_count, (unsigned long long)total);
          base = __shfl_sync(0xffffffffu, base, 31);
          unsigned long long w = base + (unsigned long long)(incl - mine);
#pragma unroll
          for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              if ((pass >> (i * 8 + j)) & 1ull) {
                const int r = (i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4);
                const int c = (j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4);
                if ((int64_t)w < A.cand_cap) {
                  A.cand_key[w] = ((uint64_t)(row0 + r) << 32) | (uint64_t)(col0 + c);
                  A.cand_sim[w] = h[i][j];
                }
                ++w;
              }
            }
          }
        }
        __syncthreads();  // accumulator cleared
      }
    }
    __syncthreads();  // staging buffers are rewritten by the next unit
  }
}

}  // namespace

int tiles_fp32_max_grid() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Opts the kernel into its dynamic shared memory once per device (outside
// any stream capture when called ahead of it).
cuapss_status tiles_fp32_init() {
  static std::mutex mu;
  static uint64_t done = 0;  // bit per device
  int dev = 0;
  CU_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && ((done >> dev) & 1ull)) return CUAPSS_OK;
  CU_TRY(cudaFuncSetAttribute(k_tiles_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kSmemBytes));
  if (dev < 64) done |= 1ull << dev;
  return CUAPSS_OK;
}

cuapss_status launch_tiles_fp32(const TileArgs& a, int grid, cudaStream_t st, bool overlap_prev) {
  ST_TRY(tiles_fp32_init());
  if (a.p % kKC != 0) return CUAPSS_EINVAL;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmemBytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = overlap_prev ? 1 : 0;
  CU_TRY(cudaLaunchKernelEx(&cfg, k_tiles_fp32, a));
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

}  // namespace cuapss
