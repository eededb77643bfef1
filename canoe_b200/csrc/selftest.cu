// selftest.cu -- a check of the bounded-wait path that the kernels use for
// their bulk copies (bulk.cuh): a wait that cannot succeed gives up after its
// spin limit and reports CANOE_EBIT_TIMEOUT instead of hanging the GPU.
// Nothing faults: the barrier's phase is completed before the kernel exits.
#include "block.cuh"
#include "bulk.cuh"

namespace cb {
namespace {

// One thread.  The mbarrier expects two arrivals; `arrivals` of them (1 or 2)
// happen before the wait, the rest after it, so that no phase is left open.
__global__ void k_bounded_wait(uint32_t *err, int spins, int arrivals) {
  __shared__ uint64_t m;
  if (threadIdx.x != 0) return;
  mbar_init(&m, 2);
  fence_mbar_init();
  for (int a = 0; a < arrivals; ++a) mbar_arrive(&m);
  if (!mbar_wait(&m, 0, spins)) atomicOr(err, (uint32_t)CANOE_EBIT_TIMEOUT);
  for (int a = arrivals; a < 2; ++a) mbar_arrive(&m);
  mbar_wait(&m, 0, spins);
}

}  // namespace
}  // namespace cb

extern "C" int canoe_selftest_bounded_wait(int spins, int complete, uint32_t *h_bits) {
  using namespace cb;
  if (!h_bits || spins < 1 || spins > (1 << 20)) {
    set_error("canoe_selftest_bounded_wait: spins in 1..2^20 and a result pointer");
    return CANOE_ERR_ARG;
  }
  uint32_t *d = nullptr;
  CB_CUDA(cudaMalloc(&d, sizeof(uint32_t)));
  cudaError_t e = cudaMemset(d, 0, sizeof(uint32_t));
  if (e == cudaSuccess) {
    k_bounded_wait<<<1, 32>>>(d, spins, complete ? 2 : 1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(h_bits, d, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(d);
  CB_CUDA(e);
  return 0;
}
