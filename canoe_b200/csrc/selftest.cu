// selftest.cu -- a check of the bounded-wait path that the kernels use for
// their bulk copies (bulk.cuh): a wait that cannot succeed gives up after its
// spin limit and reports CANOE_EBIT_TIMEOUT instead of hanging the GPU.
// Nothing faults: the barrier's phase is completed before the kernel exits.
#include "block.cuh"
#include "bulk.cuh"
#include "mlp.cuh"

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

// ---------------------------------------------------------------------------
// The same for the tensor-core completion wait of the warm-start inference
// (mlp.cuh): one warpgroup allocates TMEM, issues the layer-2 MMAs on zero
// operands and commits them to its mbarrier when `issue` is set, and waits a
// bounded number of polls.  Without the MMAs nothing can complete the phase:
// the wait must give up with CANOE_EBIT_TIMEOUT, and the columns are freed
// safely because nothing is in flight.  With them the wait must succeed and
// the accumulator must read back as zeros (CANOE_EBIT_NAN otherwise).

namespace cb {
namespace {

__global__ void __launch_bounds__(kUmmaM, 1) k_umma_wait(uint32_t *err, int spins, int issue) {
  __shared__ __align__(128) uint8_t a[kUmmaABytes];
  __shared__ __align__(128) uint8_t b[kUmmaBBytes];
  __shared__ uint64_t bar;
  __shared__ uint32_t tm_slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int q = tid; q < kUmmaABytes / 16; q += kUmmaM) reinterpret_cast<uint4 *>(a)[q] = zero;
  for (int q = tid; q < kUmmaBBytes / 16; q += kUmmaM) reinterpret_cast<uint4 *>(b)[q] = zero;
  if (warp == 0) {
    tmem_alloc(&tm_slot, (uint32_t)kMlpH);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tm_slot;
  if (tid == 0 && issue) {
    const uint32_t a0 = smem_addr(a), b0 = smem_addr(b);
    for (int ks = 0; ks < kMlpH / 16; ++ks)
      umma_bf16(tm, umma_desc(a0 + ks * 2 * (kUmmaM * 16), kUmmaM * 16, 128),
                umma_desc(b0 + ks * 2 * (kMlpH * 16), kMlpH * 16, 128), kUmmaIdesc,
                ks > 0 ? 1u : 0u);
    umma_commit(&bar);
  }
  const bool done = __syncthreads_and(mbar_wait(&bar, 0, spins));
  if (!done && tid == 0) atomicOr(err, (uint32_t)CANOE_EBIT_TIMEOUT);
  tc_fence_after();
  if (done) {
    uint32_t r[16];
    tmem_ld16(tm + ((uint32_t)(32 * warp) << 16), r);
    bool nz = false;
#pragma unroll
    for (int j = 0; j < 16; ++j) nz = nz || r[j] != 0u;
    if (nz) atomicOr(err, (uint32_t)CANOE_EBIT_NAN);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tm, (uint32_t)kMlpH);
  }
}

}  // namespace
}  // namespace cb

extern "C" int canoe_selftest_umma_wait(int spins, int issue, uint32_t *h_bits) {
  using namespace cb;
  if (!h_bits || spins < 1 || spins > (1 << 20)) {
    set_error("canoe_selftest_umma_wait: spins in 1..2^20 and a result pointer");
    return CANOE_ERR_ARG;
  }
  uint32_t *d = nullptr;
  CB_CUDA(cudaMalloc(&d, sizeof(uint32_t)));
  cudaError_t e = cudaMemset(d, 0, sizeof(uint32_t));
  if (e == cudaSuccess) {
    k_umma_wait<<<1, kUmmaM>>>(d, spins, issue ? 1 : 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(h_bits, d, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(d);
  CB_CUDA(e);
  return 0;
}

// ---------------------------------------------------------------------------
// Non-tensor FMA throughput of this GPU (the denominator for FP64 / FP32
// arithmetic): eight independent fused multiply-add chains per thread on
// every SM, long enough that launch overhead is negligible.

namespace cb {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = T(threadIdx.x + c) * T(1e-3);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
  }
  T s = x[0];
#pragma unroll
  for (int c = 1; c < 8; ++c) s += x[c];
  if (s == T(-1)) out[blockIdx.x] = s;  // keeps the chains live; never true
}

template <typename T>
int fma_peak(int iters, double *tflops) {
  int dev = 0, nsm = 0;
  CB_CUDA(cudaGetDevice(&dev));
  CB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int grid = nsm * 8, threads = 256;
  T *d = nullptr;
  CB_CUDA(cudaMalloc(&d, grid * sizeof(T)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const T a = T(0.999999), b = T(1e-7);
  k_fma_peak<T><<<grid, threads>>>(d, iters / 8, a, b);  // warm-up
  cudaEventRecord(e0);
  k_fma_peak<T><<<grid, threads>>>(d, iters, a, b);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  CB_CUDA(e);
  *tflops = 2.0 * 8.0 * (double)iters * grid * threads / (ms * 1e-3) / 1e12;
  return 0;
}

}  // namespace
}  // namespace cb

extern "C" int canoe_measure_fma_peak(int fp32, double *h_tflops) {
  using namespace cb;
  if (!h_tflops) {
    set_error("canoe_measure_fma_peak: null result pointer");
    return CANOE_ERR_ARG;
  }
  return fp32 ? fma_peak<float>(1 << 17, h_tflops) : fma_peak<double>(1 << 14, h_tflops);
}
