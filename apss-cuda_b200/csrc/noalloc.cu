// cuapss_feature_remap_noalloc: the frequency remap (posting counts, then
// features ordered by count descending, id ascending) without any device
// allocation, for callers that cannot call cudaMalloc.
//
// Who cannot allocate: a process whose device memory is already owned by
// another allocator (a framework's caching allocator that reserved the HBM
// up front, a serving process with a fixed memory budget, where a stray
// cudaMalloc fails or evicts), and code on a latency path where cudaMalloc
// and cudaFree are not allowed because they can synchronize the whole
// device. Such callers own the inputs and the outputs; all other memory this
// entry point needs lives in one file-scope device array.
//
// Scratch: g_remap_scratch below, kNoAllocScratchBytes (about 1.6 MB), sized
// for d <= kNoAllocMaxFeatures (65,536) features; larger d is rejected with
// CUAPSS_EINVAL. The array exists on every device this library's module is
// loaded on, until the process exits. Host code never hands the array's name
// to a kernel (in host code that name is a host-side shadow, not a device
// address): every call, with its device current, looks up the device address
// with cudaGetSymbolAddress (return code checked), so a reset device or a
// recreated primary context never leaves a stale address behind. The first
// call on a device can load the module, so it should come before any stream
// capture. Every call waits for its own work before it returns (it reads an
// error flag back), so the host is blocked until the remap is done. The array
// keeps the last call's contents; each call clears what must start at zero
// (the error flag and the caller's counts array). Calls whose GPU work
// overlaps (two streams, two host threads, two contexts on one device) share
// the array and race: serialise them. When a call returns CUAPSS_EINVAL after
// its launches (a bad column id or an unsorted row), perm and counts hold
// partial results and must not be used.
#include <cuda_runtime.h>

#include <mutex>

#include "ctx.cuh"
#include "prims.cuh"

namespace cuapss {

namespace {

constexpr int64_t kNoAllocMaxFeatures = 65536;
constexpr int64_t kNoAllocMaxBlocks = kNoAllocMaxFeatures / kRsTile;       // 32 sort tiles
constexpr int64_t kNoAllocHist = 256 * kNoAllocMaxBlocks;                  // 8192 bins
constexpr int64_t kNoAllocScanParts = (kNoAllocHist + kScanTile - 1) / kScanTile;

// scratch layout (bytes, 256-aligned pieces)
constexpr size_t kOffKeysA = 0;
constexpr size_t kOffKeysB = kOffKeysA + 8 * kNoAllocMaxFeatures;
constexpr size_t kOffValsA = kOffKeysB + 8 * kNoAllocMaxFeatures;
constexpr size_t kOffValsB = kOffValsA + 4 * kNoAllocMaxFeatures;
constexpr size_t kOffHist = kOffValsB + 4 * kNoAllocMaxFeatures;
constexpr size_t kOffParts = kOffHist + 4 * kNoAllocHist;
constexpr size_t kOffFlags = kOffParts + 256 * ((4 * kNoAllocScanParts + 255) / 256);
constexpr size_t kNoAllocScratchBytes = kOffFlags + 256;  // about 1.6 MB

static __device__ __align__(256) unsigned char g_remap_scratch[kNoAllocScratchBytes];

constexpr int kThreads = 256;

__global__ void k_na_check_rowptr(const int64_t* __restrict__ rp, int64_t n, int64_t nnz,
                                  int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = rp[i];
    bool bad = v < 0 || v > nnz || (i == 0 && v != 0) || (i == n && v != nnz) ||
               (i < n && rp[i + 1] < v);
    if (bad) atomicOr(err, 1);
  }
}

// One warp per row: ids in range and ascending; posting counts.
__global__ void k_na_count(const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                           int64_t n, int64_t d, int32_t* __restrict__ counts, int* err) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t lo = rp[i], hi = rp[i + 1];
    for (int64_t e = lo + lane; e < hi; e += 32) {
      const int32_t c = col[e];
      if (c < 0 || c >= d || (e > lo && col[e - 1] >= c)) {
        atomicOr(err, 1);
        continue;
      }
      atomicAdd(&counts[c], 1);
    }
  }
}

__global__ void k_na_keys(const int32_t* __restrict__ counts, int64_t d, int64_t max_count,
                          int fbits, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < d;
       f += (int64_t)gridDim.x * blockDim.x) {
    keys[f] = ((uint64_t)(max_count - counts[f]) << fbits) | (uint64_t)f;
    vals[f] = (uint32_t)f;
  }
}

__global__ void k_na_perm(const uint32_t* __restrict__ sorted_f, int64_t d,
                          int32_t* __restrict__ perm) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < d;
       r += (int64_t)gridDim.x * blockDim.x)
    perm[sorted_f[r]] = (int32_t)r;
}

inline unsigned grid_for(int64_t work) {
  int64_t g = ceil_div(work > 0 ? work : 1, kThreads);
  return (unsigned)(g < 148 * 8 ? g : 148 * 8);
}

// Device address of the scratch array on the current device, looked up on
// every call (cheap once the module is loaded).
cuapss_status scratch_for(int dev, unsigned char** out) {
  if (dev < 0) return CUAPSS_EINVAL;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_remap_scratch);
  if (e != cudaSuccess || !p) {
    record_cuda_error(e, "cudaGetSymbolAddress(g_remap_scratch)", __FILE__, __LINE__);
    return CUAPSS_ECUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return CUAPSS_OK;
}

// Exclusive scan of the (<= kNoAllocHist) histogram entries in place, with
// the block partials in scratch (one level suffices at this size).
cuapss_status scan_hist(uint32_t* hist, int64_t m, uint32_t* parts, cudaStream_t st) {
  const int64_t nb = ceil_div(m, kScanTile);
  if (nb == 1) {
    k_scan_apply<uint32_t><<<1, kScanThreads, 0, st>>>(hist, hist, m, nullptr, nullptr);
    LAUNCH_CHECK();
    return CUAPSS_OK;
  }
  k_scan_reduce<uint32_t><<<(unsigned)nb, kScanThreads, 0, st>>>(hist, m, parts);
  LAUNCH_CHECK();
  k_scan_apply<uint32_t><<<1, kScanThreads, 0, st>>>(parts, parts, nb, nullptr, nullptr);
  LAUNCH_CHECK();
  k_scan_apply<uint32_t><<<(unsigned)nb, kScanThreads, 0, st>>>(hist, hist, m, parts, nullptr);
  LAUNCH_CHECK();
  return CUAPSS_OK;
}

}  // namespace

}  // namespace cuapss

using namespace cuapss;

extern "C" cuapss_status cuapss_feature_remap_noalloc(cuapss_ctx* c, const cuapss_csr* x,
                                                      int32_t* perm, int32_t* counts) {
  if (!c || !x || !perm || !counts) return CUAPSS_EINVAL;
  if (!x->on_device) return CUAPSS_EINVAL;  // host input would need a staging copy
  if (x->n < 0 || x->d < 1 || x->nnz < 0 || !x->rowptr || (x->nnz > 0 && !x->col))
    return CUAPSS_EINVAL;
  if (x->d > kNoAllocMaxFeatures || x->n >= INT32_MAX) return CUAPSS_EINVAL;  // beyond scratch
  CU_TRY(cudaSetDevice(c->device));
  unsigned char* base = nullptr;
  ST_TRY(scratch_for(c->device, &base));
  cudaStream_t st = c->stream;
  const int64_t n = x->n, d = x->d, nnz = x->nnz;
  uint64_t* ka = reinterpret_cast<uint64_t*>(base + kOffKeysA);
  uint64_t* kb = reinterpret_cast<uint64_t*>(base + kOffKeysB);
  uint32_t* va = reinterpret_cast<uint32_t*>(base + kOffValsA);
  uint32_t* vb = reinterpret_cast<uint32_t*>(base + kOffValsB);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + kOffHist);
  uint32_t* parts = reinterpret_cast<uint32_t*>(base + kOffParts);
  int* err = reinterpret_cast<int*>(base + kOffFlags);
  // everything that must start at zero
  CU_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  CU_TRY(cudaMemsetAsync(counts, 0, sizeof(int32_t) * d, st));
  k_na_check_rowptr<<<grid_for(n + 1), kThreads, 0, st>>>(x->rowptr, n, nnz, err);
  LAUNCH_CHECK();
  int h_err = 0;
  CU_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  if (h_err) return CUAPSS_EINVAL;
  k_na_count<<<grid_for(n * 32), kThreads, 0, st>>>(x->rowptr, x->col, n, d, counts, err);
  LAUNCH_CHECK();
  CU_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  if (h_err) return CUAPSS_EINVAL;
  // LSD radix sort of (count desc, id asc) keys, ping-pong in scratch
  const int fbits = bits_for((uint64_t)d);
  const int nbits = fbits + bits_for((uint64_t)n);
  k_na_keys<<<grid_for(d), kThreads, 0, st>>>(counts, d, n, fbits, ka, va);
  LAUNCH_CHECK();
  const int nblocks = (int)ceil_div(d, kRsTile);
  for (int shift = 0; shift < nbits; shift += 8) {
    k_rs_upsweep<<<nblocks, kRsThreads, 0, st>>>(ka, d, shift, hist, nblocks);
    LAUNCH_CHECK();
    ST_TRY(scan_hist(hist, (int64_t)nblocks * 256, parts, st));
    k_rs_downsweep<<<nblocks, kRsThreads, 0, st>>>(ka, va, kb, vb, d, shift, hist, nblocks);
    LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  k_na_perm<<<grid_for(d), kThreads, 0, st>>>(va, d, perm);
  LAUNCH_CHECK();
  CU_TRY(cudaStreamSynchronize(st));
  return CUAPSS_OK;
}
