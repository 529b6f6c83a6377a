// Self-check of the bounded device waits the tile kernels rely on for
// failure detection (cuapss_selftest_bounded_wait): a kernel waits, with the
// same mbarrier try-wait primitive and a poll limit, on a barrier that
// nothing completes. The wait must give up, the kernel must report
// kErrTimeout through the error flag and return, and the context must stay
// usable. No trap, no fault: every poll is bounded.
#include <cuda_runtime.h>

#include "ctx.cuh"
#include "ptx.cuh"

namespace cuapss {
namespace {

__global__ void k_wait_for_nothing(uint32_t max_polls, int* err, uint32_t* polls_done) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival completes phase 0; none ever comes
    fence_mbar_init();
  }
  __syncthreads();
  bool done = false;
  uint32_t i = 0;
  for (; i < max_polls && !done; ++i) done = mbar_try_wait(&bar, 0);
  if (threadIdx.x == 0) {
    *polls_done = i;
    if (!done) atomicOr(err, kErrTimeout);
  }
}

}  // namespace
}  // namespace cuapss

using namespace cuapss;

extern "C" cuapss_status cuapss_selftest_bounded_wait(cuapss_ctx* c, int32_t max_polls,
                                                      int32_t* polls_done) {
  if (!c || max_polls < 1 || max_polls > (int32_t)kMaxPolls) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  int* err = nullptr;
  uint32_t* polls = nullptr;
  ST_TRY(c->ws.get("selftest:err", 1, &err));
  ST_TRY(c->ws.get("selftest:polls", 1, &polls));
  CU_TRY(cudaMemsetAsync(err, 0, sizeof(int), c->stream));
  k_wait_for_nothing<<<1, 32, 0, c->stream>>>((uint32_t)max_polls, err, polls);
  LAUNCH_CHECK();
  int h_err = 0;
  uint32_t h_polls = 0;
  CU_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaMemcpyAsync(&h_polls, polls, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  if (polls_done) *polls_done = (int32_t)h_polls;
  return (h_err & kErrTimeout) ? CUAPSS_ETIMEOUT : CUAPSS_ECUDA;
}
