// Shared host/device helpers for the CuAPSS library.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>

#include "cuapss.h"
#include <nvtx3/nvToolsExt.h>

namespace cuapss {

// Returns CUAPSS_ECUDA (after recording the message) when a CUDA call fails.
#define CU_TRY(expr)                                          \
  do {                                                        \
    cudaError_t e__ = (expr);                                 \
    if (e__ != cudaSuccess) {                                 \
      ::cuapss::record_cuda_error(e__, #expr, __FILE__, __LINE__); \
      return e__ == cudaErrorMemoryAllocation ? CUAPSS_ENOMEM : CUAPSS_ECUDA; \
    }                                                         \
  } while (0)

// Checks a kernel launch and counts it (cuapss_stats.launches).
#define LAUNCH_CHECK()                                  \
  do {                                                  \
    CU_TRY(cudaGetLastError());                         \
    ::cuapss::g_launches.fetch_add(1, std::memory_order_relaxed); \
  } while (0)

#define ST_TRY(expr)                         \
  do {                                       \
    cuapss_status s__ = (expr);              \
    if (s__ != CUAPSS_OK) return s__;        \
  } while (0)

extern std::atomic<int64_t> g_launches;

void record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
const char* last_error_message();

// Device error flags (bit mask) written by kernels.
enum : int {
  kErrRowptr = 1,      // rowptr not monotone / out of [0, nnz] / rowptr[0] != 0
  kErrColRange = 2,    // feature id outside [0, d)
  kErrColOrder = 4,    // feature ids not strictly ascending within a row
  kErrValue = 8,       // non-finite value
  kErrNorm = 16,       // | ||x|| - 1 | > tol
  kErrTimeout = 32,    // a bounded wait gave up
  kErrInternal = 64,   // an internal capacity check failed
};

constexpr int kBlockRows = 128;  // rows per row block (tile edge)
// The J side's tail postings are kept per segment of kJSegRows rows (kJSegs
// per row block), each sorted by feature: the tile kernels run a tile's tail
// one segment (a slab of kJSegRows tile columns) at a time.
constexpr int kJSegRows = 32;
constexpr int kJSegs = kBlockRows / kJSegRows;
// Tail staging capacity of the tile kernels: a block's feature groups are
// staged in shared memory in chunks of at most this many groups / postings.
// Tail postings of a row block are bucketed by the low kTailBucketBits bits
// of the tail feature (see tail.cuh).
constexpr int kTailBucketBits = 12;
constexpr uint32_t kTailBuckets = 1u << kTailBucketBits;

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline int bits_for(uint64_t v) {  // bits needed to represent values < v+1
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

// Grow-only named device buffers owned by a context; avoids cudaMalloc on
// every call.
class Workspace {
 public:
  ~Workspace() { release(); }
  // Returns a device pointer with at least `bytes` bytes (256-byte aligned).
  cuapss_status get(const std::string& name, size_t bytes, void** out) {
    if (bytes == 0) bytes = 256;
    auto it = bufs_.find(name);
    if (it != bufs_.end() && it->second.size >= bytes) {
      *out = it->second.ptr;
      return CUAPSS_OK;
    }
    if (it != bufs_.end()) {
      cudaFree(it->second.ptr);
      bufs_.erase(it);
    }
    void* p = nullptr;
    size_t want = bytes + bytes / 8;  // headroom against regrowth
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      e = cudaMalloc(&p, bytes);
      want = bytes;
      if (e != cudaSuccess) {
        cudaGetLastError();
        return CUAPSS_ENOMEM;
      }
    }
    bufs_[name] = {p, want};
    *out = p;
    return CUAPSS_OK;
  }
  template <typename T>
  cuapss_status get(const std::string& name, size_t count, T** out) {
    void* p = nullptr;
    cuapss_status s = get(name, count * sizeof(T), &p);
    *out = static_cast<T*>(p);
    return s;
  }
  size_t bytes_held() const {
    size_t s = 0;
    for (auto& kv : bufs_) s += kv.second.size;
    return s;
  }
  void release() {
    for (auto& kv : bufs_) cudaFree(kv.second.ptr);
    bufs_.clear();
  }
  // Frees the buffers whose names start with prefix.
  void release_prefix(const std::string& prefix) {
    for (auto it = bufs_.begin(); it != bufs_.end();) {
      if (it->first.compare(0, prefix.size(), prefix) == 0) {
        cudaFree(it->second.ptr);
        it = bufs_.erase(it);
      } else {
        ++it;
      }
    }
  }

 private:
  struct Buf {
    void* ptr;
    size_t size;
  };
  std::map<std::string, Buf> bufs_;
};

// NVTX ranges of a call's host-side stages (prepare, tiles, finalize), for
// Nsight timelines; without a tool attached they cost a few instructions.
// The current stage's range ends when the next begins or at scope exit.
class StageRange {
 public:
  explicit StageRange(const char* name) { nvtxRangePushA(name); }
  void next(const char* name) {
    nvtxRangePop();
    nvtxRangePushA(name);
  }
  ~StageRange() { nvtxRangePop(); }
  StageRange(const StageRange&) = delete;
  StageRange& operator=(const StageRange&) = delete;
};

}  // namespace cuapss
