// Validation, frequency remap, head block and inverted-list
// build for one join operand.
//
// Reference counterparts (fengyilin118/APSS-CUDA):
//  - per-row head norm pre_norm (main.cu:308-312, 324-325): FP64 sum of
//    squares of the head entries, here computed on the device for both the
//    head and the tail of each row, after the frequency remap;
//  - inverted index: generate_index_ptr4 (similarity_search.cu:105-191)
//    counts postings with atomics, the host scans the counts (1168-1186) and
//    construct_Index2 (221-274) scatters through an atomic cursor, so list
//    order is nondeterministic. Here the tail postings are sorted by
//    (feature, row) with an LSD radix sort and the list pointers come from a
//    device exclusive scan of the counts: lists are deterministic and sorted
//    by row (the canonical form of the reference's index);
//  - the reference fixes the head to feature ids < 4096 (similarity_search.cu
//    :130, 250, 454, 890, ...); here features are first ranked by frequency
//    and the head is the p most frequent ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "prep.cuh"
#include "prims.cuh"
#include "tail.cuh"

namespace cuapss {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_or(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void k_check_rowptr(const int64_t* __restrict__ rp, int64_t n, int64_t nnz, int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = rp[i];
    int bad = 0;
    if (v < 0 || v > nnz) bad = 1;
    if (i == 0 && v != 0) bad = 1;
    if (i == n && v != nnz) bad = 1;
    if (i < n && rp[i + 1] < v) bad = 1;
    if (bad) atomicOr(err, kErrRowptr);
  }
}

// One warp per row: id range/order, finite values, FP64 norm, posting counts.
// Hot Zipf features would serialize on their global counters, so counts are
// first gathered per CTA in shared memory and added to the global counts
// once per CTA:
//   kHistDirect: d <= kHistMax, one shared counter per feature;
//   kHistHashed: larger d, a shared hash table of kHashSlots (feature,
//     count) slots, open addressing with kHashProbes probes; the hot features
//     take their slots early and stay there, an entry whose probes all find
//     other features goes to its global counter;
//   kHistGlobal: global atomics only (small inputs).
constexpr int64_t kHistMax = 50176;
constexpr int kHashBits = 14;
constexpr int kHashSlots = 1 << kHashBits;  // 128 KB: keys + counts
constexpr int kHashProbes = 4;
constexpr uint32_t kHashEmpty = 0xffffffffu;
enum HistMode { kHistGlobal = 0, kHistDirect = 1, kHistHashed = 2 };

__device__ __forceinline__ void hist_add(int mode, int* hist, int32_t* __restrict__ counts,
                                         int32_t c) {
  if (mode == kHistDirect) {
    atomicAdd(&hist[c], 1);
    return;
  }
  if (mode == kHistHashed) {
    uint32_t* hk = reinterpret_cast<uint32_t*>(hist);
    int* hc = hist + kHashSlots;
    const uint32_t h = ((uint32_t)c * 2654435761u) >> (32 - kHashBits);
#pragma unroll
    for (int q = 0; q < kHashProbes; ++q) {
      const uint32_t slot = (h + (uint32_t)q) & (kHashSlots - 1u);
      uint32_t k = hk[slot];
      if (k == kHashEmpty) k = atomicCAS(&hk[slot], kHashEmpty, (uint32_t)c);
      if (k == kHashEmpty || k == (uint32_t)c) {
        atomicAdd(&hc[slot], 1);
        return;
      }
    }
  }
  atomicAdd(&counts[c], 1);
}

template <int MODE>
__global__ void k_check_rows(const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                             const float* __restrict__ val, int64_t n, int64_t d, float tol,
                             int check, int32_t* __restrict__ counts, int* err,
                             unsigned long long* nrm_max_bits) {
  extern __shared__ int hist[];
  if (MODE == kHistDirect) {
    for (int64_t f = threadIdx.x; f < d; f += blockDim.x) hist[f] = 0;
    __syncthreads();
  } else if (MODE == kHistHashed) {
    for (int k = threadIdx.x; k < kHashSlots; k += blockDim.x) {
      hist[k] = (int)kHashEmpty;
      hist[kHashSlots + k] = 0;
    }
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  double nrm_max = 0.0;  // this warp's rows (one global atomic per warp at the end)
  int bad_all = 0;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t lo = rp[i], hi = rp[i + 1];
    double ss = 0.0;
    int bad = 0;
    for (int64_t e = lo + lane; e < hi; e += 32) {
      const int32_t c = col[e];
      const float v = val[e];
      if (c < 0 || c >= d) bad |= kErrColRange;
      if (e > lo && col[e - 1] >= c) bad |= kErrColOrder;
      if (!isfinite(v)) bad |= kErrValue;
      ss += (double)v * (double)v;
      if (counts && c >= 0 && c < d) hist_add(MODE, hist, counts, c);
    }
    ss = warp_sum_d(ss);
    bad = warp_or(bad);
    const double nrm = sqrt(ss);
    if (check && hi > lo && fabs(nrm - 1.0) > (double)tol) bad |= kErrNorm;
    bad_all |= bad;
    nrm_max = fmax(nrm_max, nrm);
  }
  if (lane == 0) {
    if (bad_all) atomicOr(err, bad_all);
    if (nrm_max > 0.0) atomicMax(nrm_max_bits, (unsigned long long)__double_as_longlong(nrm_max));
  }
  if (MODE == kHistDirect) {
    __syncthreads();
    if (counts)
      for (int64_t f = threadIdx.x; f < d; f += blockDim.x)
        if (hist[f]) atomicAdd(&counts[f], hist[f]);
  } else if (MODE == kHistHashed) {
    __syncthreads();
    if (counts)
      for (int k = threadIdx.x; k < kHashSlots; k += blockDim.x)
        if (hist[kHashSlots + k]) atomicAdd(&counts[hist[k]], hist[kHashSlots + k]);
  }
}

__global__ void k_feat_keys(const int32_t* __restrict__ counts, int64_t d, int64_t max_count,
                            int fbits, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < d;
       f += (int64_t)gridDim.x * blockDim.x) {
    keys[f] = ((uint64_t)(max_count - counts[f]) << fbits) | (uint64_t)f;
    vals[f] = (uint32_t)f;
  }
}

__global__ void k_perm_from_sorted(const uint32_t* __restrict__ sorted_f, int64_t d,
                                   int32_t* __restrict__ perm) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < d;
       r += (int64_t)gridDim.x * blockDim.x)
    perm[sorted_f[r]] = (int32_t)r;
}

// out[r] = posting count of the feature of rank r (sorted_f: ids in rank
// order, or null for the identity order), r < m.
__global__ void k_rank_counts(const uint32_t* __restrict__ sorted_f,
                              const int32_t* __restrict__ counts, int64_t m,
                              int32_t* __restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x)
    out[r] = counts[sorted_f ? (int64_t)sorted_f[r] : r];
}

__global__ void k_iota_i32(int32_t* v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int32_t)i;
}

// Tail-balanced row blocks. One warp per caller row: its probed tail
// non-zeros (features of rank in [p, rare_from): the rare features above
// are paired explicitly, not probed) into a sort key {count << rbits | row}.
__global__ void k_row_tail_keys(const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                                const int32_t* __restrict__ perm, int64_t n, int p,
                                int64_t rare_from, int rbits, uint64_t* __restrict__ keys,
                                uint32_t* __restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    int cnt = 0;
    for (int64_t e = rp[i] + lane; e < rp[i + 1]; e += 32) {
      const int64_t r = perm[col[e]];
      cnt += r >= p && r < rare_from ? 1 : 0;
    }
    cnt = warp_sum_i(cnt);
    if (lane == 0) {
      keys[i] = ((uint64_t)cnt << rbits) | (uint64_t)i;
      vals[i] = (uint32_t)i;
    }
  }
}

// Places the rows, sorted by probed tail non-zeros ascending (sorted[k]),
// into row blocks: the R = n - 128 F lightest rows fill the last, partial
// block; the others are dealt to the F full blocks in snake order (round r
// gives block b its (r F + b)-th row, or (r F + F - 1 - b)-th in odd rounds),
// so every full block's tail is near the mean. Within a block the rows stay
// in round order, lightest first. (Dealing to the 32-row J segments instead,
// which evens the tile kernels' tail slabs, measured 1-28% slower on the
// n = d = 1M and n = 800k shapes.) rowperm[new] = caller row; newlen[new] =
// its length.
__global__ void k_deal_rows(const uint32_t* __restrict__ sorted, const int64_t* __restrict__ rp,
                            int64_t n, int64_t F, int32_t* __restrict__ rowperm,
                            int64_t* __restrict__ newlen) {
  const int64_t R = n - F * kBlockRows;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    int64_t pos;
    if (k < R) {
      pos = F * kBlockRows + k;
    } else {
      const int64_t kk = k - R, r = kk / F, q = kk % F;
      const int64_t blk = (r & 1) ? F - 1 - q : q;
      pos = blk * kBlockRows + r;
    }
    const uint32_t old = sorted[k];
    rowperm[pos] = (int32_t)old;
    newlen[pos] = rp[old + 1] - rp[old];
  }
}

// Entries of rank >= rare_from (features that occur in few rows) are neither
// head nor tail: they go, remapped, to the front of the row's range (a
// prefix of length rcount[r]) and their pairs are enumerated explicitly.
//
// One warp per row, one pass over the caller's CSR: feature ids remapped to
// their frequency rank; the head entries (rank < p) scattered straight into
// the dense head block (BF16 tiles in the tensor core's swizzled layout,
// and/or FP32 k-major slices) and summed into the FP64 head norm; the tail
// entries (rank >= p) written, remapped, to the end of the row's range in
// col2/val2 (a suffix of length tcount[r]; the head part of col2/val2 is not
// written); per-row nnz, head length and the block's largest nnz. Rows keep
// the caller's order. Nothing downstream depends on the order inside the
// tail suffix: the tail lists are built by sorts on (block, feature) and
// (J segment, feature).
//
// BF16 tile layout: one 16 KB tile per (row block, 64-feature chunk); row rr
// of the tile occupies bytes [128 rr, 128 rr + 128) and its 16-byte chunk c
// (features 8c..8c+7 of the chunk) sits at chunk position c ^ (rr % 8), the
// 128-byte swizzle the tensor core expects, so a plain bulk copy lands a tile
// in shared memory ready for tcgen05.mma. FP32 layout: head32[b][f][rr].
__global__ void k_split_rows(const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                             const float* __restrict__ val, const int32_t* __restrict__ perm,
                             const int32_t* __restrict__ rowperm,
                             const int64_t* __restrict__ rp_out, int64_t n, int p,
                             int32_t* __restrict__ col2,
                             float* __restrict__ val2, int32_t* __restrict__ hlen,
                             int32_t* __restrict__ nnz_row, float* __restrict__ hnorm,
                             int64_t* __restrict__ tcount, int32_t* __restrict__ blk_maxnnz,
                             __nv_bfloat16* __restrict__ head16, int nkc,
                             float* __restrict__ head32, int64_t rare_from,
                             int64_t* __restrict__ rcount) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t src = rowperm ? (int64_t)rowperm[i] : i;  // the caller's row at place i
    const int64_t lo = rp[src], hi = rp[src + 1];
    const int64_t olo = rp_out[i], ohi = rp_out[i + 1];  // this row's range in col2/val2
    const int64_t b = i / kBlockRows, rr = i % kBlockRows;
    int64_t nh = 0, nt = 0, nr = 0;
    double hs = 0.0;
    for (int64_t base = lo; base < hi; base += 32) {
      const int64_t e = base + lane;
      const bool valid = e < hi;
      const int32_t rank = valid ? perm[col[e]] : 0;
      const float v = valid ? val[e] : 0.0f;
      const bool head = valid && rank < p;
      const bool rare = valid && (int64_t)rank >= rare_from;
      const unsigned tb = __ballot_sync(0xffffffffu, valid && !head && !rare);
      const unsigned rb = __ballot_sync(0xffffffffu, rare);
      if (head) {
        hs += (double)v * (double)v;
        if (head16) {
          const int kc = rank >> 6, c = (rank >> 3) & 7, w = rank & 7;
          const int64_t off =
              (((b * nkc + kc) * kBlockRows + rr) * 128 + ((c ^ (int)(rr & 7)) * 16)) / 2 + w;
          head16[off] = __float2bfloat16_rn(v);
        }
        if (head32) head32[(b * p + rank) * kBlockRows + rr] = v;
      } else if (rare) {
        const int64_t dst = olo + nr + __popc(rb & lt);
        col2[dst] = rank;
        val2[dst] = v;
      } else if (valid) {
        const int64_t dst = ohi - 1 - (nt + __popc(tb & lt));
        col2[dst] = rank;
        val2[dst] = v;
      }
      nh += __popc(__ballot_sync(0xffffffffu, head));
      nt += __popc(tb);
      nr += __popc(rb);
    }
    hs = warp_sum_d(hs);
    if (lane == 0) {
      hlen[i] = (int32_t)nh;
      nnz_row[i] = (int32_t)(hi - lo);
      hnorm[i] = __double2float_ru(sqrt(hs));
      tcount[i] = nt;
      if (rcount) rcount[i] = nr;
      atomicMax(&blk_maxnnz[b], (int32_t)(hi - lo));
    }
  }
}

// Block-local lists are ordered by (bucket = f mod 2^12, tag = f >> 12):
// the fb-bit feature rotated so that its low 12 bits lead (a bijection, so
// equal features stay contiguous).
__device__ __forceinline__ uint32_t tail_rot(uint32_t f, int fb) {
  return fb > kTailBucketBits
             ? ((f & (kTailBuckets - 1u)) << (fb - kTailBucketBits)) | (f >> kTailBucketBits)
             : f;
}
__device__ __forceinline__ uint32_t tail_unrot(uint32_t k, int fb) {
  return fb > kTailBucketBits
             ? ((k & ((1u << (fb - kTailBucketBits)) - 1u)) << kTailBucketBits) |
                   (k >> (fb - kTailBucketBits))
             : k;
}

// One warp per new row: tail entries in row order (entry -> CSR index,
// row in block, value, tail feature), posting counts per tail feature and,
// when given, radix sort keys for the block-local lists (block, bucket,
// tag), the J-segment lists (J segment, feature) and the global lists
// (feature, row).
__global__ void k_tail_entries(const int64_t* __restrict__ rp2, const int32_t* __restrict__ col2,
                               const float* __restrict__ val2, const int32_t* __restrict__ hlen,
                               const int64_t* __restrict__ tptr, int64_t n, int p, int rbits,
                               int fb, uint32_t* __restrict__ tk, uint8_t* __restrict__ tr,
                               float* __restrict__ tu, uint32_t* __restrict__ tf,
                               uint64_t* __restrict__ ckeys,
                               uint32_t* __restrict__ cvals, uint64_t* __restrict__ bkeys,
                               uint32_t* __restrict__ bvals, uint64_t* __restrict__ hkeys,
                               uint32_t* __restrict__ hvals, int32_t* __restrict__ ccount) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    // the tail entries are the suffix of the row's range (tptr counts them)
    const int64_t hi = rp2[r + 1], lo = hi - (tptr[r + 1] - tptr[r]);
    const int64_t t0 = tptr[r];
    const uint64_t blk = (uint64_t)(r / kBlockRows);
    const uint64_t hblk = (uint64_t)(r / kJSegRows);
    for (int64_t k = lo + lane; k < hi; k += 32) {
      const int64_t t = t0 + (k - lo);
      const int32_t f = col2[k] - p;
      tk[t] = (uint32_t)k;
      tr[t] = (uint8_t)(r % kBlockRows);
      tu[t] = val2[k];
      tf[t] = (uint32_t)f;
      if (bkeys) {
        bkeys[t] = (blk << fb) | (uint64_t)tail_rot((uint32_t)f, fb);
        bvals[t] = (uint32_t)t;
        hkeys[t] = (hblk << fb) | (uint64_t)f;
        hvals[t] = (uint32_t)t;
      }
      if (ckeys) {
        ckeys[t] = ((uint64_t)f << rbits) | (uint64_t)r;
        cvals[t] = (uint32_t)t;
      }
      atomicAdd(&ccount[f], 1);
    }
  }
}

// I-side postings in (block, bucket, tag, row) order: key {bucket << 15 |
// tag << 7 | row in block}, value, and at the first posting of each
// feature's run the run's length (a run is one feature of one block, at most
// kBlockRows postings; 0 elsewhere).
__global__ void k_bil_fill(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                           const uint8_t* __restrict__ tr, const float* __restrict__ tu, int64_t T,
                           int fb, uint32_t* __restrict__ bil_key, float* __restrict__ bil_u,
                           uint8_t* __restrict__ bil_len) {
  const uint64_t fmask = (1ull << fb) - 1ull;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < T;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = keys[k];
    const uint32_t t = vals[k];
    const uint32_t f = tail_unrot((uint32_t)(key & fmask), fb);
    bil_key[k] = ((f & (kTailBuckets - 1u)) << 15) | ((f >> kTailBucketBits) << 7) | (uint32_t)tr[t];
    bil_u[k] = tu[t];
    int len = 0;
    if (k == 0 || keys[k - 1] != key) {
      int64_t m = k + 1;
      while (m < T && m - k < kBlockRows && keys[m] == key) ++m;
      len = (int)(m - k);
    }
    bil_len[k] = (uint8_t)len;
  }
}

// Packed J-side postings in (J segment, feature, row) order.
__global__ void k_rec_fill(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                           const uint8_t* __restrict__ tr, const float* __restrict__ tu, int64_t T,
                           uint64_t fmask, uint2* __restrict__ rec) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < T;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t t = vals[k];
    const uint32_t f = (uint32_t)(keys[k] & fmask);
    rec[k] = make_uint2((f << 8) | (uint32_t)tr[t], __float_as_uint(tu[t]));
  }
}

// ---- per-segment sorts in shared memory ----
// The block-local lists and the J-segment lists are orders of contiguous
// row-order segments (an I block's tail entries, a J segment's) by keys
// that are unique inside the segment (a feature occurs once per row), so the
// sorted order is unique: one CTA sorts a segment in shared memory with a
// stable LSD radix sort and writes the postings directly. The result equals
// the stable global radix sort by (segment, key) that is used when a segment
// exceeds kSegMax entries.
constexpr int kSegMax = 16384;   // entries per segment sorted in shared memory
constexpr int kSegThreads = 1024;
// Size classes of the segments: shared-memory capacity (entries) and threads
// per CTA, so that small segments run many CTAs per SM.
constexpr int kSegClasses = 3;
constexpr int kSegCap[kSegClasses] = {1024, 4096, kSegMax};
constexpr int kSegThr[kSegClasses] = {128, 256, kSegThreads};
constexpr int kSegBins = 512;    // digits of up to 9 bits

// Shared memory of a segment sort with NT threads and cap entries:
// keys K[cap], values V[cap], per-warp digit counters [NT/32][kSegBins],
// digit starts [kSegBins].
constexpr size_t seg_smem_bytes(int nt, int cap) {
  return (size_t)cap * 8 + (size_t)(nt / 32) * kSegBins * 4 + (size_t)kSegBins * 4;
}

// Stable LSD radix sort of (K, V)[0, len) by key bits [0, bits), len <= NT * E,
// in passes of equal digits of at most 9 bits. Between passes the elements
// live in registers: warp w holds positions [32 E w, 32 E (w + 1)) in chunks
// of 32 lanes (position order = the order so far), ranks each chunk's digits
// with match_any against per-warp counters, and the block scatters through
// the one shared buffer: digit start + the count of that digit in earlier
// warps + earlier in this warp.
template <int NT, int E>
__device__ __forceinline__ void seg_radix_sort(uint32_t* K, uint32_t* V, uint32_t* wcnt,
                                               uint32_t* dstart, int len, int bits) {
  constexpr int NW = NT / 32;
  constexpr int BPT = kSegBins / NT > 0 ? kSegBins / NT : 1;  // digits per thread (max)
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int passes = bits <= 0 ? 0 : (bits + 8) / 9;
  const int rb = passes ? (bits + passes - 1) / passes : 0;
  const int bins = 1 << rb;
  const uint32_t dmask = (uint32_t)bins - 1u;
  const int bpt = (bins + NT - 1) / NT;
  static_assert(E % 2 == 0 && NT * E <= 65536, "ranks are packed two per register");
  uint32_t key[E], val[E], rank2[E / 2];  // rank of chunk c in bits 16 (c & 1) of rank2[c / 2]
  for (int pass = 0, shift = 0; pass < passes; ++pass, shift += rb) {
    for (int i = threadIdx.x; i < NW * kSegBins; i += NT) wcnt[i] = 0;
#pragma unroll
    for (int c = 0; c < E; ++c) {
      const int idx = w * 32 * E + c * 32 + lane;
      const bool valid = idx < len;
      key[c] = valid ? K[idx] : 0u;
      val[c] = valid ? V[idx] : 0u;
    }
    __syncthreads();
    uint32_t* mine = wcnt + w * kSegBins;
#pragma unroll
    for (int c = 0; c < E; ++c) {
      const bool valid = w * 32 * E + c * 32 + lane < len;
      const unsigned vmask = __ballot_sync(0xffffffffu, valid);
      uint32_t before = 0, peers = 0;
      const uint32_t d = (key[c] >> shift) & dmask;
      if (valid) {
        peers = __match_any_sync(vmask, d);
        before = mine[d];
      }
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) mine[d] = before + __popc(peers);
      __syncwarp();
      const uint32_t r = before + __popc(peers & lt);
      if (c & 1) rank2[c / 2] |= r << 16;
      else rank2[c / 2] = r;
    }
    __syncthreads();
    // per digit: each warp's offset inside the digit, the digit's total;
    // then the exclusive scan of the totals over digits
    uint32_t dtot[BPT];
    uint32_t tsum = 0;
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
      const int d = threadIdx.x * bpt + k;
      uint32_t run = 0;
      if (k < bpt && d < bins) {
        for (int ww = 0; ww < NW; ++ww) {
          const uint32_t t = wcnt[ww * kSegBins + d];
          wcnt[ww * kSegBins + d] = run;
          run += t;
        }
      }
      dtot[k] = run;
      tsum += run;
    }
    uint32_t total;
    uint32_t start = block_excl_scan<uint32_t, NT>(tsum, &total);
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
      const int d = threadIdx.x * bpt + k;
      if (k < bpt && d < bins) {
        dstart[d] = start;
        start += dtot[k];
      }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < E; ++c) {
      if (w * 32 * E + c * 32 + lane < len) {
        const uint32_t d = (key[c] >> shift) & dmask;
        const uint32_t pos = dstart[d] + mine[d] + ((rank2[c / 2] >> (16 * (c & 1))) & 0xffffu);
        K[pos] = key[c];
        V[pos] = val[c];
      }
    }
    __syncthreads();
  }
}

// Loads the segment [s0, s0 + len) as (key(t), value bits) pairs and sorts
// it by the low `bits` bits of the keys.
template <int NT, int E, typename KeyOf>
__device__ __forceinline__ void seg_load_sort(uint32_t* smem, int cap, int64_t s0, int len,
                                              int bits, const float* __restrict__ tu, KeyOf key) {
  uint32_t* K = smem;
  uint32_t* V = smem + cap;
  uint32_t* wcnt = smem + 2 * cap;
  uint32_t* dstart = wcnt + (NT / 32) * kSegBins;
  for (int i = threadIdx.x; i < len; i += NT) {
    K[i] = key(s0 + i);
    V[i] = __float_as_uint(tu[s0 + i]);
  }
  __syncthreads();
  seg_radix_sort<NT, E>(K, V, wcnt, dstart, len, bits);
}

// Non-empty segments of ptr (nseg segments, host copy) grouped by size
// class, uploaded to ids; first[c] .. first[c + 1] are class c's entries.
inline cuapss_status seg_classes(const std::vector<int64_t>& ptr, int nseg, Workspace& ws,
                                 const std::string& tag, cudaStream_t st, int32_t** ids,
                                 int (&first)[kSegClasses + 1]) {
  std::vector<int32_t> h;
  h.reserve((size_t)nseg);
  for (int c = 0; c < kSegClasses; ++c) {
    first[c] = (int)h.size();
    const int64_t lo = c == 0 ? 0 : kSegCap[c - 1];
    for (int i = 0; i < nseg; ++i) {
      const int64_t len = ptr[i + 1] - ptr[i];
      if (len > lo && len <= kSegCap[c]) h.push_back(i);
    }
  }
  first[kSegClasses] = (int)h.size();
  ST_TRY(ws.get(tag, std::max<size_t>(h.size(), 1), ids));
  if (!h.empty())
    CU_TRY(cudaMemcpyAsync(*ids, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice,
                           st));
  return CUAPSS_OK;
}

// I-side postings of one 128-row block (one CTA per block of the list
// ids): sort key {rotated feature << 7 | row in block}; writes bil_key,
// bil_u, bil_len in the layout of k_bil_fill.
template <int NT, int E>
__global__ void __launch_bounds__(NT) k_bil_seg(const int32_t* __restrict__ ids,
                                                const int64_t* __restrict__ bptr,
                                                const uint32_t* __restrict__ tf,
                                                const uint8_t* __restrict__ tr,
                                                const float* __restrict__ tu, int fb,
                                                uint32_t* __restrict__ bil_key,
                                                float* __restrict__ bil_u,
                                                uint8_t* __restrict__ bil_len) {
  extern __shared__ uint32_t seg_sm[];
  constexpr int cap = NT * E;
  const uint32_t* K = seg_sm;
  const uint32_t* V = seg_sm + cap;
  const int b = ids[blockIdx.x];
  const int64_t s0 = bptr[b];
  const int len = (int)(bptr[b + 1] - s0);
  if (len <= 0) return;
  seg_load_sort<NT, E>(seg_sm, cap, s0, len, fb + 7, tu,
                       [&](int64_t t) { return (tail_rot(tf[t], fb) << 7) | (uint32_t)tr[t]; });
  for (int i = threadIdx.x; i < len; i += NT) {
    const uint32_t k = K[i], rf = k >> 7;
    const uint32_t f = tail_unrot(rf, fb);
    bil_key[s0 + i] =
        ((f & (kTailBuckets - 1u)) << 15) | ((f >> kTailBucketBits) << 7) | (k & 127u);
    bil_u[s0 + i] = __uint_as_float(V[i]);
    int run = 0;
    if (i == 0 || (K[i - 1] >> 7) != rf) {
      int m = i + 1;
      while (m < len && (K[m] >> 7) == rf) ++m;
      run = m - i;
    }
    bil_len[s0 + i] = (uint8_t)run;
  }
}

// J-side postings of one kJSegRows-row segment (one CTA per segment of the
// list ids): sort key {feature << 5 | row in segment}; writes records in the
// layout of k_rec_fill.
template <int NT, int E>
__global__ void __launch_bounds__(NT) k_rec_seg(const int32_t* __restrict__ ids,
                                                const int64_t* __restrict__ hptr,
                                                const uint32_t* __restrict__ tf,
                                                const uint8_t* __restrict__ tr,
                                                const float* __restrict__ tu, int fb,
                                                uint2* __restrict__ rec) {
  extern __shared__ uint32_t seg_sm[];
  constexpr int cap = NT * E;
  const uint32_t* K = seg_sm;
  const uint32_t* V = seg_sm + cap;
  const int h = ids[blockIdx.x];
  const int64_t s0 = hptr[h];
  const int len = (int)(hptr[h + 1] - s0);
  if (len <= 0) return;
  static_assert(kJSegRows == 32, "row in segment: 5 bits");
  seg_load_sort<NT, E>(seg_sm, cap, s0, len, fb + 5, tu,
                       [&](int64_t t) { return (tf[t] << 5) | ((uint32_t)tr[t] & 31u); });
  const uint32_t seg0 = (uint32_t)(h % kJSegs) * kJSegRows;  // first block row of the segment
  for (int i = threadIdx.x; i < len; i += NT) {
    const uint32_t k = K[i];
    rec[s0 + i] = make_uint2(((k >> 5) << 8) | seg0 | (k & 31u), V[i]);
  }
}

__global__ void k_seg_ptrs(const int64_t* __restrict__ tptr, int64_t n, int nh,
                           int64_t* __restrict__ hptr) {
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h <= nh;
       h += (int64_t)gridDim.x * blockDim.x)
    hptr[h] = tptr[min(n, (int64_t)h * kJSegRows)];
}

__global__ void k_block_ptrs(const int64_t* __restrict__ tptr, int64_t n, int nb,
                             int64_t* __restrict__ bptr) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= nb;
       b += (int64_t)gridDim.x * blockDim.x)
    bptr[b] = tptr[min(n, b * kBlockRows)];
}

__global__ void k_csc_fill(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                           const uint32_t* __restrict__ tk, const float* __restrict__ val2,
                           int64_t T, uint64_t rmask, uint2* __restrict__ csc,
                           uint32_t* __restrict__ entpos) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < T;
       m += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t t = vals[m];
    csc[m] = make_uint2((uint32_t)(keys[m] & rmask), __float_as_uint(val2[tk[t]]));
    entpos[t] = (uint32_t)m;
  }
}

__global__ void k_tail_products(const int32_t* __restrict__ ccount, int64_t nf,
                                unsigned long long* out) {
  unsigned long long s = 0;
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf;
       f += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long L = (unsigned long long)ccount[f];
    s += L * (L > 0 ? L - 1 : 0) / 2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}




__global__ void k_widen_i32(const int32_t* __restrict__ a, int64_t* __restrict__ b, int64_t m) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

inline unsigned grid_for(int64_t work, int per_block) {
  int64_t g = ceil_div(std::max<int64_t>(work, 1), per_block);
  return (unsigned)std::min<int64_t>(g, 148 * 32);
}

// Dynamic shared memory of the segment sorts of size class C (every class
// above 48 KB needs the opt-in; it is set for all of them).
template <int C>
cuapss_status seg_sort_attr() {
  constexpr int NT = kSegThr[C], E = kSegCap[C] / kSegThr[C];
  const int sm = (int)seg_smem_bytes(NT, kSegCap[C]);
  CU_TRY(cudaFuncSetAttribute(k_bil_seg<NT, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CU_TRY(cudaFuncSetAttribute(k_rec_seg<NT, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  return CUAPSS_OK;
}

// Kernel attributes of the segment sorts (their shared memory), once per
// device.
cuapss_status seg_sort_init() {
  static std::mutex mu;
  static uint64_t done = 0;  // bit per device
  int dev = 0;
  CU_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 64 && ((done >> dev) & 1ull)) return CUAPSS_OK;
  ST_TRY(seg_sort_attr<0>());
  ST_TRY(seg_sort_attr<1>());
  ST_TRY(seg_sort_attr<2>());
  static_assert(kSegClasses == 3, "one attribute call per size class");
  if (dev < 64) done |= 1ull << dev;
  return CUAPSS_OK;
}

// Segment sorts of size class C: the I blocks' lists and the J segments'
// records whose lengths fall in the class.
template <int C>
cuapss_status launch_seg_sorts(const int32_t* idsB, const int (&fB)[kSegClasses + 1],
                               const int32_t* idsH, const int (&fH)[kSegClasses + 1], Side& s,
                               const uint32_t* tf, int fb, cudaStream_t st) {
  constexpr int NT = kSegThr[C], E = kSegCap[C] / kSegThr[C];
  static_assert(NT * E == kSegCap[C], "class capacity");
  const size_t sm = seg_smem_bytes(NT, kSegCap[C]);
  if (fB[C + 1] > fB[C]) {
    k_bil_seg<NT, E><<<fB[C + 1] - fB[C], NT, sm, st>>>(idsB + fB[C], s.bptr, tf, s.tr, s.tu, fb,
                                                       s.bil_key, s.bil_u, s.bil_len);
    LAUNCH_CHECK();
  }
  if (fH[C + 1] > fH[C]) {
    k_rec_seg<NT, E><<<fH[C + 1] - fH[C], NT, sm, st>>>(idsH + fH[C], s.hptr, tf, s.tr, s.tu, fb,
                                                       s.bil_rec);
    LAUNCH_CHECK();
  }
  return CUAPSS_OK;
}

// ---- explicit pairs of rare features ----
// A feature that occurs in at most a few rows is a waste to probe: its J
// postings meet the I blocks' staged lists of almost every tile for nothing.
// Its pairs are enumerated instead: the rare entries are sorted by (feature,
// row); every pair of postings of one feature gives a record {fixed-point
// product << 32 | row in I block << 7 | column in J block}, grouped by
// triangular tile index, so that a tile adds its records to its tail
// accumulator directly. The grouping is a counting sort done per tile row:
// one CTA per I block walks the pairs whose first row lies in the block,
// counts them per J block in shared memory, and after a scan of the counts
// over all tiles places them from shared-memory cursors, so that each CTA
// writes one contiguous range. The order of records within a tile is not
// fixed: the accumulator's integer additions do not depend on it.

// One warp per row: its rare entries (the row's prefix) as sort keys
// {rare feature << rbits | row}, their row-major index as the payload, and
// their value bits in row-major order.
__global__ void k_rare_keys(const int64_t* __restrict__ rp2, const int32_t* __restrict__ col2,
                            const float* __restrict__ val2, const int64_t* __restrict__ rptr,
                            int64_t n, int64_t rare_from, int rbits, uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ idx, uint32_t* __restrict__ vrm) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const int64_t o = rptr[r], m = rptr[r + 1] - o, lo = rp2[r];
    for (int64_t k = lane; k < m; k += 32) {
      keys[o + k] = ((uint64_t)(col2[lo + k] - rare_from) << rbits) | (uint64_t)r;
      idx[o + k] = (uint32_t)(o + k);
      vrm[o + k] = __float_as_uint(val2[lo + k]);
    }
  }
}

// After the sort: vs[k] = value of sorted posting k, inv[row-major index] = k.
__global__ void k_rare_gather(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ vrm,
                              int64_t m, uint32_t* __restrict__ vs, uint32_t* __restrict__ inv) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t i = idx[k];
    vs[k] = vrm[i];
    inv[i] = (uint32_t)k;
  }
}

// Pairs that sorted posting k opens: the later postings of its feature (a
// feature has at most max_run postings; binary search for the end of its
// run). The total is added to *total.
__global__ void k_rare_pair_counts(const uint64_t* __restrict__ keys, int64_t m, int rbits,
                                   int max_run, int32_t* __restrict__ cnt,
                                   unsigned long long* __restrict__ total) {
  unsigned long long sum = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t f = keys[k] >> rbits;
    int64_t lo = k + 1, hi = k + max_run < m ? k + max_run : m;  // run end in [lo, hi]
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((keys[mid] >> rbits) == f) lo = mid + 1;
      else hi = mid;
    }
    cnt[k] = (int32_t)(lo - k - 1);
    sum += (unsigned long long)(lo - k - 1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0 && sum) atomicAdd(total, sum);
}

constexpr int kRareTileChunk = 8192;  // J blocks per CTA: 32 KB of counters
constexpr int kRareThreads = 512;
constexpr int kRarePhase = 1024;      // J blocks whose records a CTA places at a time
constexpr int kRareProgress = 8192;   // postings per row block with progress in shared memory

// CTA (I, y): the pairs whose first row lies in row block I and whose
// second row's block J lies in [J0, J1) = [y kRareTileChunk, (y + 1)
// kRareTileChunk) from J >= I on; the tiles (I, J) of the range are
// consecutive in triangular order from tbase. Writes the range's record
// counts to ex_off. A warp takes 32 postings at a time: their headers load
// in one step, then the lanes run over each posting's pairs in turn.
__global__ void __launch_bounds__(kRareThreads)
    k_rare_tile_counts(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ inv,
                       const int32_t* __restrict__ cnt, const int64_t* __restrict__ rptr,
                       int64_t n, int rbits, int64_t nb, int shard, int nshards,
                       uint32_t* __restrict__ ex_off) {
  __shared__ uint32_t sm[kRareTileChunk];
  const int64_t I = blockIdx.x;
  const int64_t J0 = max(I, (int64_t)blockIdx.y * kRareTileChunk);
  const int64_t J1 = min(nb, ((int64_t)blockIdx.y + 1) * kRareTileChunk);
  if (J0 >= J1) return;  // the whole CTA: a range below the diagonal
  const int nj = (int)(J1 - J0);
  const int64_t tbase = tile_index(I, J0, nb);
  if (I % nshards != shard) {  // another shard's tile row: no records here
    for (int j = threadIdx.x; j < nj; j += blockDim.x) ex_off[tbase + j] = 0u;
    return;
  }
  for (int j = threadIdx.x; j < nj; j += blockDim.x) sm[j] = 0u;
  __syncthreads();
  const uint64_t rmask = (1ull << rbits) - 1ull;
  const int64_t rlo = J0 * kBlockRows, rhi = J1 * kBlockRows;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int64_t lo = rptr[I * kBlockRows], hi = rptr[min(n, (I + 1) * kBlockRows)];
  for (int64_t i0 = lo + 32 * warp; i0 < hi; i0 += 32 * nw) {
    uint32_t k = 0;
    int c = 0;
    if (i0 + lane < hi) {
      k = inv[i0 + lane];
      c = cnt[k];
    }
    unsigned todo = __ballot_sync(0xffffffffu, c > 0);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t kk = __shfl_sync(0xffffffffu, k, src);
      const int cc = __shfl_sync(0xffffffffu, c, src);
      for (int q = lane; q < cc; q += 32) {
        const int64_t rb = (int64_t)(keys[kk + 1 + q] & rmask);
        if (rb >= rlo && rb < rhi) atomicAdd(&sm[(int)(rb / kBlockRows - J0)], 1u);
      }
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nj; j += blockDim.x) ex_off[tbase + j] = sm[j];
}

// First q in [0, c) whose row (keys[k + 1 + q]) is >= row_lo; c if none.
__device__ __forceinline__ int first_row_at(const uint64_t* __restrict__ keys, uint32_t k, int c,
                                            uint64_t rmask, int64_t row_lo) {
  int lo = 0, hi = c;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((int64_t)(keys[k + 1 + mid] & rmask) < row_lo) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

constexpr int kPlaceBatch = 4;  // postings whose first pairs load together

// Record of one pair (second posting key / value bits) at its tile's
// cursor, if the pair is valid and its second row lies below rhi (rows at
// or past rhi belong to a later phase). Returns whether it was placed.
__device__ __forceinline__ bool place_pair(bool valid, uint64_t key, uint32_t vbits, int64_t ra,
                                           float ua, uint64_t rmask, int64_t rhi, int64_t J0,
                                           uint32_t* cur, uint64_t* __restrict__ rec) {
  if (!valid) return false;
  const int64_t rb = (int64_t)(key & rmask);  // >= the phase's first row, ascending
  if (rb >= rhi) return false;
  const uint32_t at = atomicAdd(&cur[(int)(rb / kBlockRows - J0)], 1u);
  const int prod = tail_fixed(ua * __uint_as_float(vbits));
  rec[at] = ((uint64_t)(uint32_t)prod << 32) | ((uint64_t)(ra % kBlockRows) << 7) |
            (uint64_t)(rb % kBlockRows);
  return true;
}

// Dynamic shared memory of k_rare_place: the range's tile cursors, then for
// up to kRareProgress postings of the block their sorted position, pair
// count and progress.
constexpr size_t kRarePlaceSmem =
    (size_t)kRareTileChunk * 4 + (size_t)kRareProgress * (4 + 2 + 2);

// The same CTAs place every pair's record at its tile's shared-memory
// cursor (ex_off holds the tiles' first records). They do so one phase of
// kRarePhase J blocks at a time, so that the cursors being written at once,
// over all CTAs, stay few enough for their partly written sectors to wait
// in L2 until they are full. Each posting's progress (its first pair not
// yet placed; rows ascend along a feature's postings) is kept in shared
// memory, or found again by binary search in a block with more postings.
__global__ void __launch_bounds__(kRareThreads)
    k_rare_place(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vs,
                 const uint32_t* __restrict__ inv, const int32_t* __restrict__ cnt,
                 const int64_t* __restrict__ rptr, int64_t n, int rbits, int64_t nb, int shard,
                 int nshards, const uint32_t* __restrict__ ex_off, uint64_t* __restrict__ rec) {
  extern __shared__ uint8_t place_smem[];
  if ((int64_t)blockIdx.x % nshards != shard) return;  // another shard's tile row
  uint32_t* cur = reinterpret_cast<uint32_t*>(place_smem);
  uint32_t* sk = cur + kRareTileChunk;  // sorted position of each posting
  uint16_t* prog = reinterpret_cast<uint16_t*>(sk + kRareProgress);
  uint16_t* sc = prog + kRareProgress;  // its pair count (< kMaxRareCount)
  const int64_t I = blockIdx.x;
  const int64_t J0 = max(I, (int64_t)blockIdx.y * kRareTileChunk);
  const int64_t J1 = min(nb, ((int64_t)blockIdx.y + 1) * kRareTileChunk);
  if (J0 >= J1) return;  // the whole CTA: a range below the diagonal
  const int nj = (int)(J1 - J0);
  const int64_t tbase = tile_index(I, J0, nb);
  for (int j = threadIdx.x; j < nj; j += blockDim.x) cur[j] = ex_off[tbase + j];
  const uint64_t rmask = (1ull << rbits) - 1ull;
  const int64_t lo = rptr[I * kBlockRows], hi = rptr[min(n, (I + 1) * kBlockRows)];
  const bool keep = hi - lo <= kRareProgress;
  if (keep) {
    // a feature's later rows all lie past block I: only a range that starts
    // above the diagonal skips some
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      const uint32_t k = inv[i];
      const int c = cnt[k];
      sk[i - lo] = k;
      sc[i - lo] = (uint16_t)c;
      prog[i - lo] = (uint16_t)(J0 == I || c == 0 ? 0 : first_row_at(keys, k, c, rmask,
                                                                        J0 * kBlockRows));
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t P0 = J0; P0 < J1; P0 += kRarePhase) {
    const int64_t rlo = P0 * kBlockRows, rhi = min(J1, P0 + kRarePhase) * kBlockRows;
    // a warp keeps the same postings in every phase: their progress entries
    // are read and written by the same lanes
    for (int64_t i0 = lo + 32 * warp; i0 < hi; i0 += 32 * nw) {
      uint32_t k = 0;
      int c = 0, q0 = 0;
      if (i0 + lane < hi) {
        if (keep) {  // the headers of every phase after the first come from shared memory
          k = sk[i0 + lane - lo];
          c = sc[i0 + lane - lo];
          q0 = prog[i0 + lane - lo];
        } else {
          k = inv[i0 + lane];
          c = cnt[k];
          if (c > 0) q0 = first_row_at(keys, k, c, rmask, rlo);
        }
      }
      const bool live = q0 < c;
      const int64_t ra = live ? (int64_t)(keys[k] & rmask) : 0;
      const uint32_t ub = live ? vs[k] : 0u;
      unsigned todo = __ballot_sync(0xffffffffu, live);
      while (todo) {
        // kPlaceBatch postings at a time: the keys and values of their first
        // 32 pairs load together, so their latencies overlap
        int src[kPlaceBatch];
#pragma unroll
        for (int j = 0; j < kPlaceBatch; ++j) {
          src[j] = todo ? __ffs(todo) - 1 : -1;
          todo &= todo - 1;
        }
        uint32_t kk[kPlaceBatch], vb[kPlaceBatch];
        int cc[kPlaceBatch], qq[kPlaceBatch];
        int64_t rr[kPlaceBatch];
        float ua[kPlaceBatch];
        uint64_t kb[kPlaceBatch];
#pragma unroll
        for (int j = 0; j < kPlaceBatch; ++j) {
          const int sj = src[j] < 0 ? 0 : src[j];
          kk[j] = __shfl_sync(0xffffffffu, k, sj);
          cc[j] = src[j] < 0 ? 0 : __shfl_sync(0xffffffffu, c, sj);
          qq[j] = __shfl_sync(0xffffffffu, q0, sj);
          rr[j] = __shfl_sync(0xffffffffu, ra, sj);
          ua[j] = __uint_as_float(__shfl_sync(0xffffffffu, ub, sj));
          const int q = qq[j] + lane;
          kb[j] = q < cc[j] ? keys[kk[j] + 1 + q] : 0ull;
          vb[j] = q < cc[j] ? vs[kk[j] + 1 + q] : 0u;
        }
#pragma unroll
        for (int j = 0; j < kPlaceBatch; ++j) {
          if (src[j] < 0) break;  // warp-uniform
          // the lanes in the phase are a prefix: the first one out ends it
          unsigned bm = __ballot_sync(0xffffffffu, place_pair(qq[j] + lane < cc[j], kb[j], vb[j],
                                                              rr[j], ua[j], rmask, rhi, J0, cur,
                                                              rec));
          int qend = bm != 0xffffffffu ? qq[j] + __popc(bm) : cc[j];
          for (int qb = qq[j] + 32; bm == 0xffffffffu && qb < cc[j]; qb += 32) {
            const int q = qb + lane;
            const bool v = q < cc[j];
            bm = __ballot_sync(0xffffffffu,
                               place_pair(v, v ? keys[kk[j] + 1 + q] : 0ull,
                                          v ? vs[kk[j] + 1 + q] : 0u, rr[j], ua[j], rmask, rhi,
                                          J0, cur, rec));
            if (bm != 0xffffffffu) qend = qb + __popc(bm);
          }
          if (keep && lane == src[j]) prog[i0 + src[j] - lo] = (uint16_t)qend;
        }
      }
    }
  }
}

cuapss_status build_explicit_pairs(Side& s, const PrepOptions& o, int64_t* rcount, Workspace& ws,
                                   const std::string& t, cudaStream_t st) {
  const int64_t n = s.n, nb = s.nb;
  int64_t* rptr = nullptr;
  ST_TRY(ws.get(t + "rptr", (size_t)n + 1, &rptr));
  ST_TRY(exclusive_scan<int64_t>(rcount, rptr, n, rptr + n, ws, t + "rptr", st));
  int64_t m = 0;
  CU_TRY(cudaMemcpyAsync(&m, rptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  const int64_t ntiles = nb * (nb + 1) / 2;
  uint32_t* off = nullptr;
  ST_TRY(ws.get(t + "ex_off", (size_t)ntiles + 1, &off));
  s.ex_off = off;
  if (m < 2) {
    CU_TRY(cudaMemsetAsync(off, 0, sizeof(uint32_t) * (ntiles + 1), st));
    return CUAPSS_OK;
  }
  if (m >= (int64_t)UINT32_MAX - 1) return CUAPSS_EINVAL;
  const int rbits = std::max(1, bits_for((uint64_t)n));
  const int fbits = std::max(1, bits_for((uint64_t)(s.d - o.rare_from)));
  uint64_t* keys = nullptr;
  uint32_t *idx = nullptr, *vrm = nullptr, *vs = nullptr, *inv = nullptr;
  int32_t* cnt = nullptr;
  unsigned long long* total = nullptr;
  ST_TRY(ws.get(t + "rare:keys", (size_t)m, &keys));
  ST_TRY(ws.get(t + "rare:idx", (size_t)m, &idx));
  ST_TRY(ws.get(t + "rare:vrm", (size_t)m, &vrm));
  ST_TRY(ws.get(t + "rare:vs", (size_t)m, &vs));
  ST_TRY(ws.get(t + "rare:inv", (size_t)m, &inv));
  ST_TRY(ws.get(t + "rare:cnt", (size_t)m, &cnt));
  ST_TRY(ws.get(t + "rare:total", 1, &total));
  k_rare_keys<<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(s.rp2, s.col2, s.val2, rptr, n,
                                                               o.rare_from, rbits, keys, idx, vrm);
  LAUNCH_CHECK();
  ST_TRY(radix_sort_pairs(keys, idx, m, rbits + fbits, ws, t + "rare", st));
  k_rare_gather<<<grid_for(m, kThreads), kThreads, 0, st>>>(idx, vrm, m, vs, inv);
  LAUNCH_CHECK();
  CU_TRY(cudaMemsetAsync(total, 0, sizeof(unsigned long long), st));
  k_rare_pair_counts<<<grid_for(m, kThreads), kThreads, 0, st>>>(keys, m, rbits,
                                                                 o.rare_max_count, cnt, total);
  LAUNCH_CHECK();
  unsigned long long P = 0;
  CU_TRY(cudaMemcpyAsync(&P, total, sizeof(P), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  // all of the self-join's pairs; a shard keeps those of its tile rows
  if (P >= (unsigned long long)UINT32_MAX - 1) return CUAPSS_EINVAL;
  s.n_explicit = 0;
  if (P == 0) {
    CU_TRY(cudaMemsetAsync(off, 0, sizeof(uint32_t) * (ntiles + 1), st));
    return CUAPSS_OK;
  }
  const dim3 grid((unsigned)nb, (unsigned)((nb + kRareTileChunk - 1) / kRareTileChunk));
  k_rare_tile_counts<<<grid, kRareThreads, 0, st>>>(keys, inv, cnt, rptr, n, rbits, nb,
                                                    o.rare_shard, o.rare_nshards, off);
  LAUNCH_CHECK();
  ST_TRY(exclusive_scan<uint32_t>(off, off, ntiles, off + ntiles, ws, t + "ex_scan", st));
  uint32_t kept = 0;
  CU_TRY(cudaMemcpyAsync(&kept, off + ntiles, sizeof(kept), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  s.n_explicit = kept;
  if (kept == 0) return CUAPSS_OK;
  ST_TRY(ws.get(t + "ex_rec", (size_t)kept, &s.ex_rec));
  {
    static std::mutex mu;
    static uint64_t done = 0;  // attribute set, bit per device
    int dev = 0;
    CU_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 64 || !((done >> dev) & 1ull)) {
      CU_TRY(cudaFuncSetAttribute(k_rare_place, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kRarePlaceSmem));
      if (dev < 64) done |= 1ull << dev;
    }
  }
  k_rare_place<<<grid, kRareThreads, kRarePlaceSmem, st>>>(keys, vs, inv, cnt, rptr, n, rbits,
                                                          nb, o.rare_shard, o.rare_nshards, off,
                                                          s.ex_rec);
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

}  // namespace

cuapss_status validate_csr(const int64_t* rp, const int32_t* col, const float* val, int64_t n,
                           int64_t d, int64_t nnz, float tol, int check, int32_t* counts,
                           double* nrm_max, Workspace& ws, const std::string& tag,
                           cudaStream_t st) {
  int* err = nullptr;
  unsigned long long* nm = nullptr;
  ST_TRY(ws.get(tag + ":err", 1, &err));
  ST_TRY(ws.get(tag + ":nrm", 1, &nm));
  CU_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  CU_TRY(cudaMemsetAsync(nm, 0, sizeof(unsigned long long), st));
  k_check_rowptr<<<grid_for(n + 1, kThreads), kThreads, 0, st>>>(rp, n, nnz, err);
  LAUNCH_CHECK();
  int h_err = 0;
  CU_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  if (h_err) return CUAPSS_EINVAL;
  const int mode = !counts ? kHistGlobal
                   : (d <= kHistMax && nnz >= 4 * d) ? kHistDirect
                   : (d > kHistMax && nnz >= ((int64_t)1 << 22)) ? kHistHashed
                                                                  : kHistGlobal;
  if (mode != kHistGlobal) {
    static std::mutex mu;
    static uint64_t done = 0;  // attributes set, bit per device
    int dev = 0;
    CU_TRY(cudaGetDevice(&dev));
    {
      std::lock_guard<std::mutex> lk(mu);
      if (dev >= 64 || !((done >> dev) & 1ull)) {
        CU_TRY(cudaFuncSetAttribute(k_check_rows<kHistDirect>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kHistMax * sizeof(int))));
        CU_TRY(cudaFuncSetAttribute(k_check_rows<kHistHashed>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(2 * kHashSlots * sizeof(int))));
        if (dev < 64) done |= 1ull << dev;
      }
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(sms, ceil_div(n, 32)));
    if (mode == kHistDirect)
      k_check_rows<kHistDirect><<<g, 1024, (size_t)d * sizeof(int), st>>>(
          rp, col, val, n, d, tol, check, counts, err, nm);
    else
      k_check_rows<kHistHashed><<<g, 1024, 2 * kHashSlots * sizeof(int), st>>>(
          rp, col, val, n, d, tol, check, counts, err, nm);
  } else {
    k_check_rows<kHistGlobal><<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(
        rp, col, val, n, d, tol, check, counts, err, nm);
  }
  LAUNCH_CHECK();
  unsigned long long h_nm = 0;
  CU_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaMemcpyAsync(&h_nm, nm, sizeof(h_nm), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  if (h_err) return CUAPSS_EINVAL;
  double v;
  memcpy(&v, &h_nm, sizeof(v));
  if (nrm_max) *nrm_max = v;
  return CUAPSS_OK;
}

cuapss_status feature_perm(const int32_t* counts, int64_t d, int64_t max_count, int remap,
                           int32_t* perm, Workspace& ws, cudaStream_t st) {
  if (!remap) {
    k_iota_i32<<<grid_for(d, kThreads), kThreads, 0, st>>>(perm, d);
    LAUNCH_CHECK();
    return CUAPSS_OK;
  }
  uint64_t* keys = nullptr;
  uint32_t* vals = nullptr;
  ST_TRY(ws.get("perm:keys", (size_t)d, &keys));
  ST_TRY(ws.get("perm:vals", (size_t)d, &vals));
  const int fbits = bits_for((uint64_t)d);
  k_feat_keys<<<grid_for(d, kThreads), kThreads, 0, st>>>(counts, d, max_count, fbits, keys, vals);
  LAUNCH_CHECK();
  ST_TRY(radix_sort_pairs(keys, vals, d, fbits + bits_for((uint64_t)max_count), ws, "perm", st));
  k_perm_from_sorted<<<grid_for(d, kThreads), kThreads, 0, st>>>(vals, d, perm);
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

// Rare-feature statistics for candidate thresholds C[k]: out[3k] = features
// occurring in more than C[k] rows, out[3k + 1] = pairs of the features
// occurring in at most C[k] rows, out[3k + 2] = their postings.
constexpr int kRareCands = 8;
__host__ __device__ constexpr int rare_cand(int k) { return kMaxRareCount >> k; }  // 2048 .. 16

__global__ void k_rare_stats(const int32_t* __restrict__ counts, int64_t d,
                             unsigned long long* __restrict__ out) {
  unsigned long long above[kRareCands] = {}, pairs[kRareCands] = {}, posts[kRareCands] = {};
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < d;
       f += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = counts[f];
#pragma unroll
    for (int k = 0; k < kRareCands; ++k) {
      if (c > rare_cand(k)) {
        above[k] += 1ull;
      } else {
        pairs[k] += (unsigned long long)(c * (c - 1) / 2);
        posts[k] += (unsigned long long)c;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kRareCands; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      above[k] += __shfl_xor_sync(0xffffffffu, above[k], o);
      pairs[k] += __shfl_xor_sync(0xffffffffu, pairs[k], o);
      posts[k] += __shfl_xor_sync(0xffffffffu, posts[k], o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&out[3 * k], above[k]);
      atomicAdd(&out[3 * k + 1], pairs[k]);
      atomicAdd(&out[3 * k + 2], posts[k]);
    }
  }
}

cuapss_status rare_feature_candidates(const int32_t* counts, int64_t d, Workspace& ws,
                                      cudaStream_t st, std::vector<RareCandidate>* cands) {
  cands->clear();
  unsigned long long* out = nullptr;
  ST_TRY(ws.get("rare:stats", 3 * kRareCands, &out));
  CU_TRY(cudaMemsetAsync(out, 0, sizeof(unsigned long long) * 3 * kRareCands, st));
  k_rare_stats<<<grid_for(d, kThreads), kThreads, 0, st>>>(counts, d, out);
  LAUNCH_CHECK();
  unsigned long long h[3 * kRareCands];
  CU_TRY(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  for (int k = 0; k < kRareCands; ++k) {
    // the features of count <= C hold the ranks from (features above C) on
    RareCandidate c;
    c.max_count = rare_cand(k);
    c.rank = (int64_t)h[3 * k];
    c.pairs = (int64_t)h[3 * k + 1];
    c.postings = (int64_t)h[3 * k + 2];
    if (c.postings > 0) cands->push_back(c);
  }
  return CUAPSS_OK;
}

cuapss_status rank_count_prefix(const int32_t* counts, int64_t d, int remap, int64_t m,
                                Workspace& ws, cudaStream_t st, std::vector<int64_t>* prefix) {
  m = std::max<int64_t>(0, std::min(m, d));
  prefix->assign((size_t)m + 1, 0);
  if (m == 0) return CUAPSS_OK;
  uint32_t* vals = nullptr;
  if (remap) ST_TRY(ws.get("perm:vals", (size_t)d, &vals));  // ids by rank (feature_perm)
  int32_t* out = nullptr;
  ST_TRY(ws.get("perm:rank_counts", (size_t)m, &out));
  k_rank_counts<<<grid_for(m, kThreads), kThreads, 0, st>>>(remap ? vals : nullptr, counts, m, out);
  LAUNCH_CHECK();
  std::vector<int32_t> h((size_t)m);
  CU_TRY(cudaMemcpyAsync(h.data(), out, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  for (int64_t r = 0; r < m; ++r) (*prefix)[(size_t)r + 1] = (*prefix)[(size_t)r] + h[(size_t)r];
  return CUAPSS_OK;
}

cuapss_status build_side(Side& s, const PrepOptions& o, const int32_t* perm, Workspace& ws,
                         const std::string& tag, cudaStream_t st) {
  const int64_t n = s.n, d = s.d, nnz = s.nnz;
  if (n >= INT32_MAX || nnz >= (int64_t)UINT32_MAX - 1) return CUAPSS_EINVAL;
  // the dense head blocks are built in slices of 32 (FP32) or 64 (BF16)
  // features; a head wider than d is padded with zero columns
  const int64_t gran = o.want_head16 ? 64 : (o.want_head32 ? 32 : 1);
  s.p = (int)std::min<int64_t>(o.p, ceil_div(d, gran) * gran);
  const int p = s.p;
  s.nb = (int)ceil_div(n, kBlockRows);
  const int nb = s.nb;
  const int rbits = std::max(1, bits_for((uint64_t)n));
  const int fbits = std::max(1, bits_for((uint64_t)d));
  const uint64_t rmask = (1ull << rbits) - 1;
  const std::string t = tag + ":";
  // ---- row order: the caller's, or tail-balanced blocks ----
  ST_TRY(ws.get(t + "rowperm", (size_t)n, &s.rowperm));
  ST_TRY(ws.get(t + "rp2", (size_t)n + 1, &s.rp2));
  const int32_t* place = nullptr;  // new row -> caller row, null: identity
  const int64_t full_blocks = n / kBlockRows;
  if (o.balance_rows && full_blocks >= 2) {
    const int rbits = std::max(1, bits_for((uint64_t)n));
    uint64_t* keys = nullptr;
    uint32_t* vals = nullptr;
    int64_t* newlen = nullptr;
    ST_TRY(ws.get(t + "bal:keys", (size_t)n, &keys));
    ST_TRY(ws.get(t + "bal:vals", (size_t)n, &vals));
    ST_TRY(ws.get(t + "bal:len", (size_t)n + 1, &newlen));
    k_row_tail_keys<<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(
        s.rp0, s.col0, perm, n, p, o.rare_from > 0 ? o.rare_from : INT64_MAX, rbits, keys, vals);
    LAUNCH_CHECK();
    // tail counts are < 2^31: rbits + 31 key bits at most (the sort takes the
    // bits of the largest possible count, bounded by d)
    ST_TRY(radix_sort_pairs(keys, vals, n, rbits + std::max(1, bits_for((uint64_t)d)), ws,
                            t + "bal", st));
    k_deal_rows<<<grid_for(n, kThreads), kThreads, 0, st>>>(vals, s.rp0, n, full_blocks,
                                                            s.rowperm, newlen);
    LAUNCH_CHECK();
    ST_TRY(exclusive_scan<int64_t>(newlen, s.rp2, n, s.rp2 + n, ws, t + "bal:scan", st));
    place = s.rowperm;
  } else {
    k_iota_i32<<<grid_for(n, kThreads), kThreads, 0, st>>>(s.rowperm, n);
    LAUNCH_CHECK();
    CU_TRY(cudaMemcpyAsync(s.rp2, s.rp0, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToDevice,
                           st));
  }
  // ---- one pass: remap, head block, row statistics, tail suffixes ----
  ST_TRY(ws.get(t + "col2", (size_t)std::max<int64_t>(nnz, 1), &s.col2));
  ST_TRY(ws.get(t + "val2", (size_t)std::max<int64_t>(nnz, 1), &s.val2));
  int64_t* tcount = nullptr;
  int64_t* rcount = nullptr;
  if (o.rare_from > 0) ST_TRY(ws.get(t + "rcount", (size_t)n + 1, &rcount));
  s.ex_off = nullptr;
  s.ex_rec = nullptr;
  s.n_explicit = 0;
  ST_TRY(ws.get(t + "hlen", (size_t)n, &s.hlen));
  ST_TRY(ws.get(t + "nnzrow", (size_t)n, &s.nnz_row));
  ST_TRY(ws.get(t + "hnorm", (size_t)n, &s.hnorm));
  ST_TRY(ws.get(t + "tcount", (size_t)n + 1, &tcount));
  ST_TRY(ws.get(t + "blkmax", (size_t)nb + 1, &s.blk_maxnnz));
  CU_TRY(cudaMemsetAsync(s.blk_maxnnz, 0, sizeof(int32_t) * (nb + 1), st));
  s.head32 = nullptr;
  s.head16 = nullptr;
  int nkc = 0;
  if (o.want_head32 && p > 0) {
    const size_t hb = (size_t)nb * p * kBlockRows;
    ST_TRY(ws.get(t + "head32", hb, &s.head32));
    CU_TRY(cudaMemsetAsync(s.head32, 0, hb * sizeof(float), st));
  }
  if (o.want_head16 && p > 0) {
    if (p % 64 != 0) return CUAPSS_EINVAL;
    nkc = p / 64;
    const size_t hb = (size_t)nb * nkc * kBlockRows * 64;
    ST_TRY(ws.get(t + "head16", hb, &s.head16));
    CU_TRY(cudaMemsetAsync(s.head16, 0, hb * sizeof(__nv_bfloat16), st));
  }
  k_split_rows<<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(
      s.rp0, s.col0, s.val0, perm, place, s.rp2, n, p, s.col2, s.val2, s.hlen, s.nnz_row,
      s.hnorm, tcount, s.blk_maxnnz, s.head16, nkc, s.head32,
      o.rare_from > 0 ? o.rare_from : INT64_MAX, o.rare_from > 0 ? rcount : nullptr);
  LAUNCH_CHECK();
  if (o.rare_from > 0) ST_TRY(build_explicit_pairs(s, o, rcount, ws, t, st));
  ST_TRY(ws.get(t + "tptr", (size_t)n + 1, &s.tptr));
  ST_TRY(exclusive_scan<int64_t>(tcount, s.tptr, n, s.tptr + n, ws, t + "tptr", st));
  // ---- tail: segment pointers (blocks, J segments), host copies ----
  const int nh = kJSegs * nb;  // J segments, the last ones possibly empty
  ST_TRY(ws.get(t + "bptr", (size_t)nb + 1, &s.bptr));
  ST_TRY(ws.get(t + "hptr", (size_t)nh + 1, &s.hptr));
  k_block_ptrs<<<grid_for(nb + 1, kThreads), kThreads, 0, st>>>(s.tptr, n, nb, s.bptr);
  LAUNCH_CHECK();
  k_seg_ptrs<<<grid_for(nh + 1, kThreads), kThreads, 0, st>>>(s.tptr, n, nh, s.hptr);
  LAUNCH_CHECK();
  std::vector<int64_t> h_hptr((size_t)nh + 1);
  s.h_bptr.resize(nb + 1);
  CU_TRY(cudaMemcpyAsync(s.h_bptr.data(), s.bptr, sizeof(int64_t) * (nb + 1),
                         cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaMemcpyAsync(h_hptr.data(), s.hptr, sizeof(int64_t) * (nh + 1),
                         cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  s.ntail = s.h_bptr[nb];
  s.max_block_tail = 0;
  for (int b = 0; b < nb; ++b)
    s.max_block_tail = std::max<int64_t>(s.max_block_tail, s.h_bptr[b + 1] - s.h_bptr[b]);
  // segments sorted in shared memory unless one exceeds kSegMax entries
  const bool seg_sort = s.max_block_tail <= kSegMax;
  // ---- tail: entries in row order, block-local inverted lists ----
  const int64_t T = s.ntail;
  if (T >= (int64_t)UINT32_MAX - 1) return CUAPSS_EINVAL;
  const int64_t nf = std::max<int64_t>(d - p, 0);
  // I-side keys hold an 8-bit tag above the 12-bit bucket: tail features < 2^20
  if (nf > (1 << 20)) return CUAPSS_EINVAL;
  const int fb = std::max(1, bits_for((uint64_t)nf));
  const int bb = std::max(1, bits_for((uint64_t)nb));
  uint64_t *ckeys = nullptr, *bkeys = nullptr, *hkeys = nullptr;
  uint32_t *cvals = nullptr, *bvals = nullptr, *hvals = nullptr;
  int32_t* ccount = nullptr;
  ST_TRY(ws.get(t + "tk", (size_t)T, &s.tk));
  ST_TRY(ws.get(t + "tr", (size_t)T, &s.tr));
  ST_TRY(ws.get(t + "tu", (size_t)T, &s.tu));
  uint32_t* tf = nullptr;
  ST_TRY(ws.get(t + "tf", (size_t)T, &tf));
  if (!seg_sort) {
    ST_TRY(ws.get(t + "bkeys", (size_t)T, &bkeys));
    ST_TRY(ws.get(t + "bvals", (size_t)T, &bvals));
    ST_TRY(ws.get(t + "hkeys", (size_t)T, &hkeys));
    ST_TRY(ws.get(t + "hvals", (size_t)T, &hvals));
  }
  ST_TRY(ws.get(t + "ccount", (size_t)nf + 1, &ccount));
  if (o.want_csc) {
    ST_TRY(ws.get(t + "ckeys", (size_t)T, &ckeys));
    ST_TRY(ws.get(t + "cvals", (size_t)T, &cvals));
  }
  CU_TRY(cudaMemsetAsync(ccount, 0, sizeof(int32_t) * (nf + 1), st));
  k_tail_entries<<<grid_for(n * 32, kThreads), kThreads, 0, st>>>(
      s.rp2, s.col2, s.val2, s.hlen, s.tptr, n, p, rbits, fb, s.tk, s.tr, s.tu, tf, ckeys,
      cvals, bkeys, bvals, hkeys, hvals, ccount);
  LAUNCH_CHECK();
  ST_TRY(ws.get(t + "bil_key", (size_t)T, &s.bil_key));
  ST_TRY(ws.get(t + "bil_u", (size_t)T, &s.bil_u));
  ST_TRY(ws.get(t + "bil_len", (size_t)T, &s.bil_len));
  ST_TRY(ws.get(t + "bil_rec", (size_t)T, &s.bil_rec));
  if (seg_sort) {
    // block-local lists in (bucket, tag, row) order and J-segment records in
    // (feature, row) order, one CTA per segment
    if (T > 0) {
      ST_TRY(seg_sort_init());
      int32_t *idsB = nullptr, *idsH = nullptr;
      int fB[kSegClasses + 1], fH[kSegClasses + 1];
      ST_TRY(seg_classes(s.h_bptr, nb, ws, t + "segB", st, &idsB, fB));
      ST_TRY(seg_classes(h_hptr, nh, ws, t + "segH", st, &idsH, fH));
      ST_TRY(launch_seg_sorts<0>(idsB, fB, idsH, fH, s, tf, fb, st));
      ST_TRY(launch_seg_sorts<1>(idsB, fB, idsH, fH, s, tf, fb, st));
      ST_TRY(launch_seg_sorts<2>(idsB, fB, idsH, fH, s, tf, fb, st));
    }
  } else {
    // block-local inverted lists: stable sort by (block, bucket, tag) keeps
    // rows ascending inside a feature
    ST_TRY(radix_sort_pairs(bkeys, bvals, T, bb + fb, ws, t + "bil", st));
    k_bil_fill<<<grid_for(T, kThreads), kThreads, 0, st>>>(bkeys, bvals, s.tr, s.tu, T, fb,
                                                          s.bil_key, s.bil_u, s.bil_len);
    LAUNCH_CHECK();
    // J-side postings: per kJSegRows-row segment, sorted by feature, packed
    ST_TRY(radix_sort_pairs(hkeys, hvals, T, std::max(1, bits_for((uint64_t)nh)) + fb, ws,
                            t + "rec", st));
    k_rec_fill<<<grid_for(T, kThreads), kThreads, 0, st>>>(hkeys, hvals, s.tr, s.tu, T,
                                                          (1ull << fb) - 1, s.bil_rec);
    LAUNCH_CHECK();
  }
  // ---- global inverted lists (feature, row), on request ----
  if (o.want_csc) {
    uint32_t* entpos = nullptr;
    ST_TRY(ws.get(t + "entpos", (size_t)T, &entpos));
    ST_TRY(ws.get(t + "cptr", (size_t)nf + 1, &s.cptr));
    ST_TRY(ws.get(t + "csc", (size_t)T, &s.csc));
    ST_TRY(radix_sort_pairs(ckeys, cvals, T, rbits + fb, ws, t + "csc", st));
    k_csc_fill<<<grid_for(T, kThreads), kThreads, 0, st>>>(ckeys, cvals, s.tk, s.val2, T, rmask,
                                                          s.csc, entpos);
    LAUNCH_CHECK();
    int64_t* c64 = nullptr;
    ST_TRY(ws.get(t + "ccount64", (size_t)nf + 1, &c64));
    k_widen_i32<<<grid_for(nf, kThreads), kThreads, 0, st>>>(ccount, c64, nf);
    LAUNCH_CHECK();
    ST_TRY(exclusive_scan<int64_t>(c64, s.cptr, nf, s.cptr + nf, ws, t + "cptr", st));
  }
  unsigned long long* red = nullptr;
  ST_TRY(ws.get(t + "red", 2, &red));
  CU_TRY(cudaMemsetAsync(red, 0, 2 * sizeof(unsigned long long), st));
  k_tail_products<<<grid_for(nf, kThreads), kThreads, 0, st>>>(ccount, nf, red);
  LAUNCH_CHECK();
  unsigned long long hred[2] = {0, 0};
  CU_TRY(cudaMemcpyAsync(hred, red, sizeof(hred), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  s.tail_products = (int64_t)hred[0];
  return CUAPSS_OK;
}

}  // namespace cuapss
