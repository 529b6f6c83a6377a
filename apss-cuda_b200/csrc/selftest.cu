// Self-check of the bounded device waits the tile kernels rely on for
// failure detection (cuapss_selftest_bounded_wait): a kernel waits, with the
// same mbarrier wait and a device-time deadline, on a barrier that nothing
// completes. The wait must give up, the kernel must report
// kErrTimeout through the error flag and return, and the context must stay
// usable. No trap, no fault: every poll is bounded.
#include <cuda_runtime.h>

#include "ctx.cuh"
#include "ptx.cuh"

namespace cuapss {
namespace {

__global__ void k_wait_for_nothing(uint64_t limit_ns, int* err, unsigned long long* waited) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival completes phase 0; none ever comes
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t t0 = globaltimer_ns();
  const bool done = mbar_wait(&bar, 0, limit_ns);
  const uint64_t t1 = globaltimer_ns();
  if (threadIdx.x == 0) {
    *waited = (unsigned long long)(t1 - t0);
    if (!done) atomicOr(err, kErrTimeout);
  }
}

}  // namespace
}  // namespace cuapss

using namespace cuapss;

extern "C" cuapss_status cuapss_selftest_bounded_wait(cuapss_ctx* c, int32_t limit_us,
                                                      int64_t* waited_ns) {
  if (!c || limit_us < 1 || (uint64_t)limit_us * 1000ull > kWaitLimitNs) return CUAPSS_EINVAL;
  CU_TRY(cudaSetDevice(c->device));
  int* err = nullptr;
  unsigned long long* waited = nullptr;
  ST_TRY(c->ws.get("selftest:err", 1, &err));
  ST_TRY(c->ws.get("selftest:waited", 1, &waited));
  CU_TRY(cudaMemsetAsync(err, 0, sizeof(int), c->stream));
  k_wait_for_nothing<<<1, 32, 0, c->stream>>>((uint64_t)limit_us * 1000ull, err, waited);
  LAUNCH_CHECK();
  int h_err = 0;
  unsigned long long h_waited = 0;
  CU_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CU_TRY(cudaMemcpyAsync(&h_waited, waited, sizeof(h_waited), cudaMemcpyDeviceToHost,
                         c->stream));
  CU_TRY(cudaStreamSynchronize(c->stream));
  if (waited_ns) *waited_ns = (int64_t)h_waited;
  return (h_err & kErrTimeout) ? CUAPSS_ETIMEOUT : CUAPSS_ECUDA;
}
