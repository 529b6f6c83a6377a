// Mixed-precision hybrid pair-tile kernel: BF16 head on the 5th-generation
// tensor cores (tcgen05, FP32 accumulators in tensor memory), FP32 tail on
// the CUDA cores, threshold epilogue with a proven error band.
//
// Head. The p most frequent features of every 128-row block are stored as a
// dense BF16 block, pre-arranged in global memory in the 128-byte-swizzled
// K-major layout the tensor core reads, so one 16 KB bulk (TMA) copy moves a
// [128 rows x 64 features] operand tile straight into shared memory. For a
// tile (I, J): D[128 x 128] = H_I * H_J^T, accumulated in tensor memory over
// p/64 chunks (4 MMAs of K = 16 each). This replaces the reference's
// per-pair sparse-dense head dot (similarity_apss_rest / similarity_join_rest,
// fengyilin118/APSS-CUDA similarity_search.cu:441-506, 854-915).
//
// Warp roles (one CTA per SM, persistent; the producer takes units of work
// from a global counter as the CTA gets to them and publishes their ids to
// the other roles through a ring of kUnitRing slots):
//   warp 0          producer: bulk copies of I and J operand tiles into a
//                   3- or 4-stage shared-memory ring (mbarrier full/empty);
//   warp 1          MMA: allocates 256 tensor-memory columns (two 128-column
//                   accumulators), one thread issues tcgen05.mma and commits;
//   kTW tail warps  the sparse tail of each tile in fixed point (tail.cuh),
//                   one slab of kSlabCols tile columns (one J segment) at a
//                   time, into one of two shared slab accumulators;
//   kEW epilogue    two per tensor-memory lane quarter: per slab, the
//   warps           accumulator columns are read with tcgen05.ld, head +
//                   tail is compared with t - eps(i, j), candidates are
//                   compacted with a warp ballot and the slab accumulator is
//                   cleared and handed back to the tail warps.
// The tail of slab s + 1 runs while the epilogue drains slab s (and each tail
// thread's first J postings of slab s + 1 are loaded during slab s), and the MMAs
// of the next tile run while both work on this one. The hand-offs are
// mbarriers: afull (tail -> epilogue) and aempty (epilogue -> tail) per slab
// buffer, tfull (MMA -> epilogue) and tempty (epilogue -> MMA) per tensor
// memory accumulator.
// eps(i, j) bounds BF16 input rounding (2^-8 relative per factor) and the
// FP32 / fixed-point sums, so no pair with FP64 similarity >= t is dropped;
// the finalize stage decides the band exactly in FP64.
//
// Every mbarrier wait is bounded by device time; a timeout raises
// kErrTimeout and a shared abort flag that the other roles' waits poll.
// A tail or epilogue warp that gave up stops working and signalling but still
// takes part in its group's named barriers, so no warp is left waiting on
// one; the producer and MMA threads drain their in-flight copies and MMAs,
// tensor memory is freed and the kernel returns.
#include <cuda_runtime.h>

#include <mutex>

#include "ptx.cuh"
#include "tail.cuh"
#include "tiles.cuh"

namespace cuapss {

namespace {

constexpr int kTW = 22;                       // tail warps
constexpr int kEW = 8;                        // epilogue warps, 2 per tensor-memory lane quarter
constexpr int kTT = kTW * 32;                 // tail threads
constexpr int kET = kEW * 32;                 // epilogue threads
constexpr int kFirstEpi = 2 + kTW;            // first epilogue warp
constexpr int kThreads = 64 + kTT + kET;      // + producer warp + MMA warp
static_assert(kThreads == 1024, "one CTA of 32 warps per SM");
static_assert(kFirstEpi % 4 == 0, "epilogue warp w reads tensor-memory lanes 32 (w % 4) ..");
constexpr int kKC = 64;                       // BF16 features per chunk (128-byte rows)
constexpr int kTileBytes = kBlockRows * kKC * 2;  // 16 KB per operand chunk
constexpr int kSlabCols = kJSegRows;          // tile columns per slab (one J segment)
constexpr int kSlabs = kJSegs;                // slabs per tile
constexpr int kSlabInts = kBlockRows * kSlabCols;  // one slab accumulator
constexpr int kEpiCols = kSlabCols / (kEW / 4);    // slab columns per epilogue thread
static_assert(kEpiCols == 16 || kEpiCols == 32, "tensor-memory loads of 16 or 32 columns");
// Tensor-memory columns of a variant whose MMA tiles span JW J blocks: two
// accumulators of 128 x (128 JW) FP32.
template <int JW>
__host__ __device__ constexpr uint32_t tmem_cols() { return 256u * JW; }
constexpr int kTailBar = 1;
constexpr int kEpiBar = 2;
// J postings per thread per load batch: 3, or 2 when the thread also holds
// explicit rare-pair records in registers (64 registers a thread)
template <bool EX>
constexpr int batch_postings() { return EX ? 2 : 3; }
constexpr int kUnitRing = 8;                  // unit ids published ahead by the producer
constexpr int kUnitReaders = 1 + kTW + kEW;   // MMA thread + tail warps + epilogue warps
static_assert(kSlabCols == 32, "slab accumulator rows are 32 ints (8 swizzled groups)");

struct SmemM {
  uint8_t* stage;       // STAGES x (A 16 KB | B JW x 16 KB), 1024-byte aligned
  int* acc;             // [2][128][32] slab accumulators (swizzled groups)
  float* hnj;           // [2][128] per-column head margins of a tile
  uint64_t* full;
  uint64_t* empty;
  uint64_t* tfull;
  uint64_t* tempty;
  uint64_t* afull;
  uint64_t* aempty;
  uint64_t* drain;
  uint64_t* ufull;      // [kUnitRing] a unit id was published
  uint64_t* uempty;     // [kUnitRing] every role has read it
  int* uring;           // [kUnitRing] unit ids
  uint32_t* tmem_base;
  int* abort;
  TailStage ts;
};

__host__ __device__ constexpr size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Shared-memory layout of the variant with STAGES operand stages of an I
// chunk and JW J chunks, and CAP staged tail postings.
template <int STAGES, int CAP, int JW>
struct Cfg {
  static constexpr int kBars = 2 * STAGES + 2 + 2 + 2 + 2 + 1 + 2 * kUnitRing;
  static constexpr size_t kStageBytes = (size_t)(1 + JW) * kTileBytes;
  static constexpr size_t kAcc = (size_t)STAGES * kStageBytes;
  static constexpr size_t kHnj = align_up(kAcc + (size_t)2 * kSlabInts * 4, 16);
  static constexpr size_t kBar = align_up(kHnj + (size_t)2 * kBlockRows * 4, 16);
  static constexpr size_t kRing = align_up(kBar + (size_t)kBars * 8, 16);
  static constexpr size_t kTmem = align_up(kRing + (size_t)kUnitRing * 4, 16);
  static constexpr size_t kAbort = kTmem + 16;
  static constexpr size_t kTail = align_up(kAbort + 16, 16);
  static constexpr size_t kTotal = align_up(kTail + tail_stage_bytes<CAP>(), 16);
  static constexpr size_t kSmem = kTotal + 1024;  // + alignment slack
  static_assert(kSmem <= 232448, "shared memory budget");
};

template <int STAGES, int CAP, int JW>
__device__ __forceinline__ SmemM carve(uint8_t* raw) {
  using C = Cfg<STAGES, CAP, JW>;
  uint8_t* base = reinterpret_cast<uint8_t*>(align_up(reinterpret_cast<size_t>(raw), 1024));
  SmemM s;
  s.stage = base;
  s.acc = reinterpret_cast<int*>(base + C::kAcc);
  s.hnj = reinterpret_cast<float*>(base + C::kHnj);
  uint64_t* b = reinterpret_cast<uint64_t*>(base + C::kBar);
  s.full = b;
  s.empty = b + STAGES;
  s.tfull = b + 2 * STAGES;
  s.tempty = b + 2 * STAGES + 2;
  s.afull = b + 2 * STAGES + 4;
  s.aempty = b + 2 * STAGES + 6;
  s.drain = b + 2 * STAGES + 8;
  s.ufull = b + 2 * STAGES + 9;
  s.uempty = b + 2 * STAGES + 9 + kUnitRing;
  s.uring = reinterpret_cast<int*>(base + C::kRing);
  s.tmem_base = reinterpret_cast<uint32_t*>(base + C::kTmem);
  s.abort = reinterpret_cast<int*>(base + C::kAbort);
  s.ts = tail_stage_at<CAP>(base + C::kTail);
  return s;
}

// Bounded wait (kWaitLimitNs of device time) that also gives up when another
// role raised the abort flag.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity,
                                              const volatile int* abort) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 0; i < kMaxPolls; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort || globaltimer_ns() - t0 >= kWaitLimitNs) return false;
  }
  return false;
}

__device__ __forceinline__ void raise_abort(const TileArgs& A, volatile int* abort) {
  if (!*abort) {
    *abort = 1;
    atomicOr(A.err, kErrTimeout);
  }
}

// wait_or_abort for a whole warp: every lane waits (so every lane acquires
// what the arrivals released) and the warp takes one answer, so it stays
// converged for its warp-synchronous work; on a give-up the abort is raised.
// Returns the warp's new `live`.
__device__ __forceinline__ bool warp_wait(const TileArgs& A, uint64_t* bar, uint32_t parity,
                                          volatile int* abort, bool live) {
  bool got = live ? wait_or_abort(bar, parity, abort) : true;
  got = __all_sync(0xffffffffu, got);
  if (live && !got && (threadIdx.x & 31) == 0) raise_abort(A, abort);
  return live && got;
}

// First batch of a slab's J postings [k0, k1): thread tid of nthreads takes
// postings tid, tid + nthreads, ...; unused slots hold the end marker.
template <int NB>
__device__ __forceinline__ void load_batch(const TileArgs& A, int64_t k0, int64_t k1, int tid,
                                           int nthreads, uint2 (&rec)[NB]) {
  const int n = (int)(k1 - k0);
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int k = tid + q * nthreads;
    rec[q] = k < n ? __ldg(&A.bilJ_rec[k0 + k]) : make_uint2(0xffffffffu, 0u);
  }
}

template <int NB>
__device__ __forceinline__ void probe_batch(const TailStage& S, const uint2 (&rec)[NB], int* acc,
                                            int cofs) {
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    if (rec[q].x == 0xffffffffu) break;  // the rest of the batch is past the range
    tail_probe<true>(S, rec[q].x >> 8, (int)(rec[q].x & 0xffu) - cofs, __uint_as_float(rec[q].y),
                     acc, kSlabCols);
  }
}

// Thread tid's explicit rare-feature record of a tile whose records are
// [lo, hi): {row in I block << 7 | column in J block} and its fixed-point
// product, or kNoRecord.
constexpr uint32_t kNoRecord = 0xffffffffu;
__device__ __forceinline__ void load_record(const TileArgs& A, uint32_t lo, uint32_t hi, int tid,
                                            uint32_t& rc, int& rv) {
  rc = kNoRecord;
  rv = 0;
  if (lo + (uint32_t)tid < hi) {
    const uint64_t rec = __ldg(&A.ex_rec[lo + tid]);
    rc = (uint32_t)rec & 0x3fffu;
    rv = (int)(rec >> 32);
  }
}

// The postings of a slab past its first batch (long slabs only).
template <int NB>
__device__ __forceinline__ void tail_rest(const TileArgs& A, const TailStage& S, const TailI& T,
                                          int64_t k0, int64_t k1, int* acc, int cofs, int tid,
                                          int nthreads) {
  if (k1 - k0 <= (int64_t)NB * nthreads || !T.any) return;
  for (int64_t kb = k0 + (int64_t)NB * nthreads; kb < k1; kb += (int64_t)NB * nthreads) {
    uint2 rec[NB];
    load_batch<NB>(A, kb, k1, tid, nthreads, rec);
    probe_batch<NB>(S, rec, acc, cofs);
  }
}

struct MmaArgs {
  const uint8_t* headI16;
  const uint8_t* headJ16;
  int nkc;  // p / 64
};

template <int STAGES, int CAP, int JW, bool EX>
__global__ void __launch_bounds__(kThreads, 1) k_tiles_mma(const TileArgs A, const MmaArgs M) {
  extern __shared__ uint8_t smem_raw[];
  const SmemM S = carve<STAGES, CAP, JW>(smem_raw);
  constexpr size_t kStageBytes = Cfg<STAGES, CAP, JW>::kStageBytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int* abort = S.abort;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&S.tfull[b], 1);
      mbar_init(&S.tempty[b], kEW);
      mbar_init(&S.afull[b], kTW);
      mbar_init(&S.aempty[b], kEW);
    }
    mbar_init(S.drain, 1);
    for (int k = 0; k < kUnitRing; ++k) {
      mbar_init(&S.ufull[k], 1);
      mbar_init(&S.uempty[k], kUnitReaders);
    }
    *abort = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(S.tmem_base, tmem_cols<JW>());
    tmem_relinquish();
  }
  if (warp >= 2)
    for (int i = threadIdx.x - 64; i < 2 * kSlabInts; i += kTT + kET) S.acc[i] = 0;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *S.tmem_base;
  allow_dependent_launch();

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      // units are taken from a global counter as the CTA gets to them and
      // published to the other roles through the unit ring
      uint32_t it = 0;
      bool ok = true;
      for (uint32_t k = 0; ok; ++k) {
        const uint32_t slot = k % kUnitRing, ur = k / kUnitRing;
        if (!wait_or_abort(&S.uempty[slot], (ur & 1u) ^ 1u, abort)) {
          raise_abort(A, abort);
          break;
        }
        const int u = atomicAdd(A.unit_counter, 1);
        reinterpret_cast<volatile int*>(S.uring)[slot] = u;
        mbar_arrive(&S.ufull[slot]);
        if (u >= A.nunits) break;
        const int4 U = A.units[u];
        if (U.y >= U.z) continue;
        for (int J = U.y; ok && J < U.z; J += JW) {
          const int w = U.z - J < JW ? U.z - J : JW;  // J blocks of this MMA tile
          for (int kc = 0; kc < M.nkc; ++kc, ++it) {
            const uint32_t s = it % STAGES, round = it / STAGES;
            if (!wait_or_abort(&S.empty[s], (round & 1u) ^ 1u, abort)) {
              raise_abort(A, abort);
              ok = false;
              break;
            }
            uint8_t* dst = S.stage + (size_t)s * kStageBytes;
            mbar_arrive_expect_tx(&S.full[s], (uint32_t)(1 + w) * kTileBytes);
            bulk_g2s(dst, M.headI16 + ((size_t)U.x * M.nkc + kc) * kTileBytes, kTileBytes,
                     &S.full[s]);
            if (w == 2)  // the second J block's rows follow the first's
              bulk_g2s(dst + 2 * kTileBytes,
                       M.headJ16 + ((size_t)(J + 1) * M.nkc + kc) * kTileBytes, kTileBytes,
                       &S.full[s]);
            bulk_g2s(dst + kTileBytes, M.headJ16 + ((size_t)J * M.nkc + kc) * kTileBytes,
                     kTileBytes, &S.full[s]);
          }
        }
      }
      // drain: the last copies issued must have landed before the CTA exits
      const uint32_t first = it > (uint32_t)STAGES ? it - STAGES : 0u;
      for (uint32_t q = first; q < it; ++q)
        if (!mbar_wait(&S.full[q % STAGES], (q / STAGES) & 1u)) raise_abort(A, abort);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ----------------------------------------------------------------- MMA
    if (lane == 0) {
      // N = 128 w: one MMA tile spans w <= JW J blocks
      const uint32_t idesc1 = umma_idesc_bf16(kBlockRows, kBlockRows);
      const uint32_t idesc2 = umma_idesc_bf16(kBlockRows, 2 * kBlockRows);
      uint32_t it = 0, tt = 0;
      bool ok = true;
      for (uint32_t k = 0; ok; ++k) {
        const uint32_t slot = k % kUnitRing, ur = k / kUnitRing;
        if (!wait_or_abort(&S.ufull[slot], ur & 1u, abort)) {
          raise_abort(A, abort);
          break;
        }
        const int u = reinterpret_cast<volatile int*>(S.uring)[slot];
        mbar_arrive(&S.uempty[slot]);
        if (u >= A.nunits) break;
        const int4 U = A.units[u];
        if (U.y >= U.z) continue;
        for (int J = U.y; ok && J < U.z; J += JW, ++tt) {
          const int w = U.z - J < JW ? U.z - J : JW;
          const uint32_t idesc = w == 2 ? idesc2 : idesc1;
          const uint32_t b = tt & 1u, tround = tt >> 1;
          if (!wait_or_abort(&S.tempty[b], (tround & 1u) ^ 1u, abort)) {
            raise_abort(A, abort);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * (uint32_t)(kBlockRows * JW);
          for (int kc = 0; kc < M.nkc; ++kc, ++it) {
            const uint32_t s = it % STAGES, round = it / STAGES;
            if (!wait_or_abort(&S.full[s], round & 1u, abort)) {
              raise_abort(A, abort);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint8_t* st = S.stage + (size_t)s * kStageBytes;
            const uint64_t ad = umma_desc_sw128(st);
            const uint64_t bd = umma_desc_sw128(st + kTileBytes);
#pragma unroll
            for (int k = 0; k < kKC / 16; ++k)
              umma_bf16(d, ad + 2u * k, bd + 2u * k, idesc, (kc | k) != 0 ? 1u : 0u);
            umma_commit(&S.empty[s]);
          }
          if (ok) umma_commit(&S.tfull[b]);
        }
      }
      // drain: every MMA issued must be complete before tensor memory is freed
      if (it > 0) {
        umma_commit(S.drain);
        if (!mbar_wait(S.drain, 0)) raise_abort(A, abort);
      }
    }
    __syncwarp();
  } else if (warp < kFirstEpi) {
    // ------------------------------------------------------------- tail
    // Each thread keeps the first batch of the next slab's J postings in
    // registers (loaded while it works on this slab), so the load latency
    // of a slab's records overlaps the previous slab's probes.
    // The J segment pointers of the next J block are loaded one block ahead
    // (32-bit: a side holds fewer than 2^32 tail postings).
    const int ttid = threadIdx.x - 64;
    bool live = true;
    uint32_t g = 0;  // slabs processed by this CTA
    for (uint32_t ku = 0;; ++ku) {
      const uint32_t slot = ku % kUnitRing, ur = ku / kUnitRing;
      live = warp_wait(A, &S.ufull[slot], ur & 1u, abort, live);
      const int u = live ? reinterpret_cast<volatile int*>(S.uring)[slot] : A.nunits;
      __syncwarp();
      if (live && lane == 0) mbar_arrive(&S.uempty[slot]);
      // every tail warp is done with the previous unit's staging; all stop together
      if (named_bar_or(kTailBar, kTT, u >= A.nunits)) break;
      const int4 U = A.units[u];
      if (U.y >= U.z) continue;
      const int I = U.x;
      const int nch = tail_nchunks<CAP>(A, I);
      TailI T{};
      if (nch == 1) T = stage_tail_chunk<kTT, kTailBar, CAP>(A, S.ts, I, 0, ttid);
      uint32_t hc[kJSegs + 1], hn[kJSegs + 1];
#pragma unroll
      for (int m = 0; m <= kJSegs; ++m) hc[m] = (uint32_t)A.hptrJ[kJSegs * U.y + m];
      constexpr int kBatch = batch_postings<EX>();
      uint2 nxt[kBatch];
      load_batch<kBatch>(A, hc[0], hc[1], ttid, kTT, nxt);
      // explicit rare-feature records: the bounds of the current and the next
      // tile, and this thread's record of each (loaded two slabs ahead; a
      // tile's records beyond the first kTT are loaded where they are used)
      uint32_t ec0 = 0, ec1 = 0, en0 = 0, en1 = 0;
      uint32_t rc = kNoRecord, rn = kNoRecord;
      int rv = 0, rnv = 0;
      if (EX) {
        const int64_t t0 = tile_index(I, U.y, A.nbI);
        ec0 = A.ex_off[t0];
        ec1 = A.ex_off[t0 + 1];
        load_record(A, ec0, ec1, ttid, rc, rv);
      }
      for (int J = U.y; J < U.z; ++J) {
        if (J + 1 < U.z) {
#pragma unroll
          for (int m = 0; m <= kJSegs; ++m) hn[m] = (uint32_t)A.hptrJ[kJSegs * (J + 1) + m];
          if (EX) {
            const int64_t t1 = tile_index(I, J + 1, A.nbI);
            en0 = A.ex_off[t1];
            en1 = A.ex_off[t1 + 1];
          }
        }
#pragma unroll
        for (int q = 0; q < kSlabs; ++q, ++g) {
          const uint32_t k = g & 1u, use = g >> 1;
          const int64_t k0 = hc[q], k1 = hc[q + 1];
          uint2 cur[kBatch];
#pragma unroll
          for (int b = 0; b < kBatch; ++b) cur[b] = nxt[b];
          // the next slab of this unit: its first batch, in flight from here
          if (q + 1 < kSlabs) load_batch<kBatch>(A, hc[q + 1], hc[q + 2], ttid, kTT, nxt);
          else if (J + 1 < U.z) load_batch<kBatch>(A, hn[0], hn[1], ttid, kTT, nxt);
          if (EX && q == kSlabs - 2 && J + 1 < U.z) load_record(A, en0, en1, ttid, rn, rnv);
          live = warp_wait(A, &S.aempty[k], (use & 1u) ^ 1u, abort, live);
          int* acc = S.acc + k * kSlabInts;
          const int cofs = q * kSlabCols;
          if (nch == 1) {
            if (live && T.any) {
              probe_batch<kBatch>(S.ts, cur, acc, cofs);
              tail_rest<kBatch>(A, S.ts, T, k0, k1, acc, cofs, ttid, kTT);
            }
          } else {
            for (int c = 0; c < nch; ++c) {
              const TailI Tc = stage_tail_chunk<kTT, kTailBar, CAP>(A, S.ts, I, c, ttid);
              if (live && Tc.any) {
                probe_batch<kBatch>(S.ts, cur, acc, cofs);
                tail_rest<kBatch>(A, S.ts, Tc, k0, k1, acc, cofs, ttid, kTT);
              }
              named_bar(kTailBar, kTT);  // staging rewritten by the next chunk
            }
          }
          if (EX && live && rc != kNoRecord && (int)((rc & 127u) >> 5) == q)
            atomicAdd(acc + acc_cell<true>((int)(rc >> 7), (int)(rc & 31u), kSlabCols), rv);
          if (EX && live && ec1 - ec0 > (uint32_t)kTT)
            tail_explicit<true>(A, ec0 + kTT, ec1, acc, kSlabCols, cofs, kSlabCols, ttid, kTT);
          __syncwarp();
          if (live && lane == 0) mbar_arrive(&S.afull[k]);
        }
#pragma unroll
        for (int m = 0; m <= kJSegs; ++m) hc[m] = hn[m];
        ec0 = en0;
        ec1 = en1;
        rc = rn;
        rv = rnv;
      }
    }
  } else {
    // --------------------------------------------------------- epilogue
    const int ew = warp - kFirstEpi;
    const int etid = threadIdx.x - (64 + kTT);
    const int q4 = warp & 3;         // tensor-memory lane quarter of this warp
    const int colh = ew >> 2;        // which kEpiCols columns of each slab
    const int row = 32 * q4 + lane;  // tile row of this thread
    bool live = true;
    uint32_t tt = 0, g = 0, mt = 0;  // J tiles, slabs, MMA tiles of this CTA
    for (uint32_t ku = 0;; ++ku) {
      const uint32_t slot = ku % kUnitRing, ur = ku / kUnitRing;
      live = warp_wait(A, &S.ufull[slot], ur & 1u, abort, live);
      const int u = live ? reinterpret_cast<volatile int*>(S.uring)[slot] : A.nunits;
      __syncwarp();
      if (live && lane == 0) mbar_arrive(&S.uempty[slot]);
      if (named_bar_or(kEpiBar, kET, u >= A.nunits)) break;  // all stop together
      const int4 U = A.units[u];
      if (U.y >= U.z) continue;
      const int I = U.x;
      const int64_t row0 = (int64_t)I * kBlockRows;
      const int rowsI = (int)(A.nI - row0 < kBlockRows ? A.nI - row0 : kBlockRows);
      const bool row_ok = row < rowsI;
      const float hn_r = row_ok ? A.hnormI[row0 + row] : 0.0f;
      const double t_r = A.t_row ? (row_ok ? (double)A.t_row[row0 + row] : 2.0) : (double)A.t;
      for (int J = U.y; J < U.z; ++J, ++tt) {
        // J block jj of MMA tile mt (which spans up to JW J blocks)
        const int jj = (J - U.y) % JW;
        const bool mt_last = jj == JW - 1 || J + 1 == U.z;
        const uint32_t b = mt & 1u, tround = mt >> 1;
        const int64_t col0 = (int64_t)J * kBlockRows;
        const int colsJ = (int)(A.nJ - col0 < kBlockRows ? A.nJ - col0 : kBlockRows);
        const bool diag = A.self && (I == J);
        const bool simple = !diag && colsJ == kBlockRows;
        const int kmax = min(A.blkmaxI[I], A.blkmaxJ[J]);
        const float t_lo = __double2float_rd(t_r - (A.eps_c1 * kmax + A.eps_c0));
        float* hnj = S.hnj + (tt & 1u) * kBlockRows;
        if (etid < kBlockRows)
          hnj[etid] =
              etid < colsJ ? __double2float_ru(A.eps_head * (double)A.hnormJ[col0 + etid]) : 0.0f;
        named_bar(kEpiBar, kET);
        if (jj == 0) {
          live = warp_wait(A, &S.tfull[b], tround & 1u, abort, live);
          tc_fence_after();
        }
        for (int q = 0; q < kSlabs; ++q, ++g) {
          const uint32_t k = g & 1u, use = g >> 1;
          live = warp_wait(A, &S.afull[k], use & 1u, abort, live);
          if (live) {
            // ---- head (tensor memory) + tail (slab accumulator) vs t - eps
            const int cbase = q * kSlabCols + colh * kEpiCols;  // first tile column
            uint32_t v[kEpiCols];
            const uint32_t taddr = tmem + b * (uint32_t)(kBlockRows * JW) +
                                   (uint32_t)(jj * kBlockRows + cbase) +
                                   ((uint32_t)(32 * q4) << 16);
            tmem_ld(taddr, v);
            int* arow = S.acc + k * kSlabInts + row * kSlabCols;
            const float4* hn4 = reinterpret_cast<const float4*>(hnj + cbase);
            uint32_t pass = 0;
#pragma unroll
            for (int j4 = 0; j4 < kEpiCols / 4; ++j4) {
              const int grp = colh * (kEpiCols / 4) + j4;  // logical 4-column group
              int4* cell = reinterpret_cast<int4*>(arow + ((grp ^ (row & 7)) << 2));
              const int4 t4 = *cell;
              *cell = make_int4(0, 0, 0, 0);
              const float4 h4 = hn4[j4];
              const int tq[4] = {t4.x, t4.y, t4.z, t4.w};
              const float hh[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                const int j = 4 * j4 + kk;
                const int c = cbase + j;
                const float s = fmaf(__int2float_rn(tq[kk]), kTailUnscale, __uint_as_float(v[j]));
                v[j] = __float_as_uint(s);
                const float thr = __fmaf_rd(-hn_r, hh[kk], t_lo);
                bool okp = (s >= thr) && row_ok;
                if (!simple) okp = okp && (c < colsJ) && (!diag || c > row);
                pass |= (uint32_t)okp << j;
              }
            }
            if (__any_sync(0xffffffffu, pass != 0u)) {
              const int mine = __popc(pass);
              int incl = mine;
#pragma unroll
              for (int o = 1; o < 32; o <<= 1) {
                const int x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += x;
              }
              const int total = __shfl_sync(0xffffffffu, incl, 31);
              unsigned long long base = 0;
              if (lane == 31) base = atomicAdd(A.cand_count, (unsigned long long)total);
              base = __shfl_sync(0xffffffffu, base, 31);
              unsigned long long w = base + (unsigned long long)(incl - mine);
#pragma unroll
              for (int j = 0; j < kEpiCols; ++j) {
                if ((pass >> j) & 1u) {
                  if ((int64_t)w < A.cand_cap) {
                    A.cand_key[w] =
                        ((uint64_t)(row0 + row) << 32) | (uint64_t)(col0 + cbase + j);
                    A.cand_sim[w] = __uint_as_float(v[j]);
                  }
                  ++w;
                }
              }
            }
          }
          __syncwarp();
          if (live && lane == 0) mbar_arrive(&S.aempty[k]);
        }
        if (mt_last) {
          tc_fence_before();
          __syncwarp();
          if (live && lane == 0) mbar_arrive(&S.tempty[b]);
          ++mt;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, tmem_cols<JW>());
  }
}

}  // namespace

// Kernel variants, by the largest I block tail (staged postings) and whether
// the caller's plan is head-bound:
//   wide   MMA tiles of two J blocks (N = 256) over 3 stages of 48 KB: the I
//          chunk is read once per two J blocks, 24 KB of operands per
//          128 x 128 tile instead of 32 KB, 144 KB in flight; staging for
//          5,936 tail postings;
//   small  one J block per MMA tile, 4 stages of 32 KB, 7,936 postings;
//   big    one J block per MMA tile, 3 stages, 12,768 postings.
// The operand stream runs near the L2's bandwidth, so the wide variant, which
// needs fewer bytes per tile, wins where the head sets the pace (measured at
// n = 200,000 of the n = d = 1M shape: p = 1,536 58.3 ms against 72.6 ms).
// Where the tail sets the pace it loses 6-7% (n = 400,000 and 1M, p = 1,024),
// so the caller asks for it only for head-bound plans.
constexpr int kWideStages = 3, kWideCap = 5936;
constexpr int kSmallStages = 4, kSmallCap = 7936;
constexpr int kBigStages = 3, kBigCap = 12768;

template <int STAGES, int CAP, int JW>
cudaError_t set_smem_attr() {
  cudaError_t e = cudaFuncSetAttribute(k_tiles_mma<STAGES, CAP, JW, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Cfg<STAGES, CAP, JW>::kSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tiles_mma<STAGES, CAP, JW, true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Cfg<STAGES, CAP, JW>::kSmem);
}

// The kernel of variant (STAGES, CAP, JW), with or without explicit records.
template <int STAGES, int CAP, int JW>
cudaError_t launch_variant(const cudaLaunchConfig_t& cfg, const TileArgs& a, const MmaArgs& m) {
  if (a.ex_off) return cudaLaunchKernelEx(&cfg, k_tiles_mma<STAGES, CAP, JW, true>, a, m);
  return cudaLaunchKernelEx(&cfg, k_tiles_mma<STAGES, CAP, JW, false>, a, m);
}

// Opts the kernels into their dynamic shared memory once per device (outside
// any stream capture when called ahead of it).
cuapss_status tiles_mma_init() {
  static std::mutex mu;
  static uint64_t done = 0;  // bit per device
  int dev = 0;
  CU_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && ((done >> dev) & 1ull)) return CUAPSS_OK;
  CU_TRY((set_smem_attr<kWideStages, kWideCap, 2>()));
  CU_TRY((set_smem_attr<kSmallStages, kSmallCap, 1>()));
  CU_TRY((set_smem_attr<kBigStages, kBigCap, 1>()));
  if (dev < 64) done |= 1ull << dev;
  return CUAPSS_OK;
}

cuapss_status launch_tiles_mma(const TileArgs& a, const void* headI16, const void* headJ16,
                               int p, int grid, cudaStream_t st, bool overlap_prev,
                               bool head_bound) {
  ST_TRY(tiles_mma_init());
  if (p <= 0 || p % kKC != 0) return CUAPSS_EINVAL;
  MmaArgs m;
  m.headI16 = static_cast<const uint8_t*>(headI16);
  m.headJ16 = static_cast<const uint8_t*>(headJ16);
  m.nkc = p / kKC;
  const int variant = head_bound && a.max_tailI <= kWideCap ? 0
                      : a.max_tailI <= kSmallCap            ? 1
                                                            : 2;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = variant == 0   ? Cfg<kWideStages, kWideCap, 2>::kSmem
                         : variant == 1 ? Cfg<kSmallStages, kSmallCap, 1>::kSmem
                                        : Cfg<kBigStages, kBigCap, 1>::kSmem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = overlap_prev ? 1 : 0;
  if (variant == 0) CU_TRY((launch_variant<kWideStages, kWideCap, 2>(cfg, a, m)));
  else if (variant == 1) CU_TRY((launch_variant<kSmallStages, kSmallCap, 1>(cfg, a, m)));
  else CU_TRY((launch_variant<kBigStages, kBigCap, 1>(cfg, a, m)));
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

size_t tiles_mma_smem_bytes() { return Cfg<kBigStages, kBigCap, 1>::kSmem; }

}  // namespace cuapss
