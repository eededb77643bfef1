// mlp.cuh -- the warm-start network of the learned saturation adjustment:
// a 4 -> H -> H -> 1 multilayer perceptron with tanh hidden units mapping
// (density, specific internal energy, total H2O, total NH3) to the
// converged temperature.  This component has no counterpart in the
// reference: it only proposes the starting point of the Newton iteration of
// the saturation adjustment, whose tolerance and fallback are unchanged.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "bulk.cuh"

namespace cb {

constexpr int kMlpIn = 4;
constexpr int kMlpH = 64;
// parameter layout (FP32, row-major [out][in]):
//   w1[H*4] b1[H] w2[H*H] b2[H] w3[H] b3[1]
constexpr int kMlpOffW1 = 0;
constexpr int kMlpOffB1 = kMlpOffW1 + kMlpH * kMlpIn;
constexpr int kMlpOffW2 = kMlpOffB1 + kMlpH;
constexpr int kMlpOffB2 = kMlpOffW2 + kMlpH * kMlpH;
constexpr int kMlpOffW3 = kMlpOffB2 + kMlpH;
constexpr int kMlpOffB3 = kMlpOffW3 + kMlpH;
constexpr int kMlpNParams = kMlpOffB3 + 1;

// what a satadj kernel needs to run the network: FP32 parameters, BF16 copy
// of w2 (the tensor-core operand), and the input / output normalisation
struct MlpView {
  const float *p;             // kMlpNParams
  const __nv_bfloat16 *w2h;   // H*H, row-major [out][in]
  float in_mean[kMlpIn], in_istd[kMlpIn];
  float out_mean, out_std;
};

// hardware tanh approximation (PTX tanh.approx.f32)
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05).
//
// One warpgroup (128 threads) infers 128 cells at a time as one M = 128 row
// tile, one row (cell) per thread:
//   layer 1 (4 -> 64, 2 % of the flops) runs in FP32 on the CUDA cores, each
//     thread writing its row's 64 BF16 hidden values into the warpgroup's A
//     tile in shared memory;
//   layer 2 (64 -> 64) is four tcgen05.mma of K = 16, BF16 x BF16 with FP32
//     accumulation into the warpgroup's 64 tensor-memory (TMEM) columns,
//     row m in lane m;
//   the epilogue reads each thread's row back with tcgen05.ld (warp w of a
//     warpgroup reads TMEM lanes 32 w .. 32 w + 31), adds the bias, applies
//     tanh and forms layer 3's dot product in registers.
// The warpgroup's first thread issues its MMAs and commits them to the
// warpgroup's mbarrier, which its threads wait on (bounded); the warpgroup
// synchronises through its own named barrier (id 1 + warpgroup).
//
// The kernels that use it are persistent, one CTA of WG warpgroups per SM,
// the warpgroups working on their own chunks without waiting on one
// another.  On B200 a kernel holding TMEM instructions is resident at one
// CTA per SM, whatever its registers and shared memory allow (the occupancy
// query returns 1 for such a kernel and 3-5 for the same kernel without
// them), so several small CTAs per SM are not available: an 8.4 M-cell
// streaming kernel ran 0.076 ms plain, 0.31 ms with 256-thread CTAs that
// merely contain an untaken tcgen05.alloc path, 0.59 ms with 128-thread
// CTAs.  The CTA stages the weights and allocates its TMEM once
// (mlp_umma_setup), each warpgroup infers any number of chunks
// (mlp_umma_infer), and the CTA frees the columns at the end
// (mlp_umma_teardown).
//
// Operands use the no-swizzle K-major canonical layout: 8-row x 16-byte core
// matrices of 128 contiguous bytes; the 16-byte chunk holding elements
// k = 8 kc .. 8 kc + 7 of row r of a `rows`-row operand sits at
// kc * rows * 16 + (r / 8) * 128 + (r % 8) * 16.  In a shared-memory matrix
// descriptor the stride between 8-row groups (SBO) is then 128 bytes and the
// stride between the two K chunks of one MMA (LBO) rows * 16 bytes.

constexpr int kUmmaM = 128;                      // rows per tile = threads per warpgroup
constexpr int kUmmaABytes = kUmmaM * kMlpH * 2;  // one BF16 A tile, 16 KB
constexpr int kUmmaBBytes = kMlpH * kMlpH * 2;   // BF16 w2, 8 KB

// dynamic shared memory of a CTA of WG warpgroups: WG A tiles, w2, the FP32
// weights, WG mbarriers and the TMEM address
template <int WG>
struct UmmaLayout {
  static_assert(WG >= 1 && WG * kMlpH <= 512, "TMEM holds 512 columns");
  static constexpr int kThreads = WG * kUmmaM;
  static constexpr uint32_t kCols = WG * kMlpH <= 64    ? 64u
                                    : WG * kMlpH <= 128 ? 128u
                                    : WG * kMlpH <= 256 ? 256u
                                                        : 512u;  // a power of two
  static constexpr int kOffB = WG * kUmmaABytes;
  static constexpr int kOffW = kOffB + kUmmaBBytes;  // w1, b1, b2, w3 (FP32)
  static constexpr int kOffW1 = kOffW;
  static constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn * 4;
  static constexpr int kOffB2 = kOffB1 + kMlpH * 4;
  static constexpr int kOffW3 = kOffB2 + kMlpH * 4;
  static constexpr int kOffBar = kOffW3 + kMlpH * 4;
  static constexpr int kOffTmem = kOffBar + WG * 8;
  static constexpr int kBytes = kOffTmem + 16;
};

// instruction descriptor of tcgen05.mma kind::f16: FP32 D (bits 4-5 = 1),
// BF16 A (bits 7-9 = 1) and B (bits 10-12 = 1), both K-major (bits 15, 16 =
// 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28
constexpr uint32_t kUmmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                ((uint32_t)(kMlpH >> 3) << 17) | ((uint32_t)(kUmmaM >> 4) << 24);

// named-barrier reductions over `n` threads (a warpgroup): every thread
// gets the OR / AND of v
__device__ __forceinline__ bool bar_red_or(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, %3, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ bool bar_red_and(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, %2, %3, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ uint32_t umma_chunk(int r, int kc, int rows) {
  return (uint32_t)kc * (uint32_t)(rows * 16) + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u;
}

// shared-memory matrix descriptor: start address, LBO and SBO in 16-byte
// units (bits 0-13, 16-29, 32-45), descriptor version 1 (bits 46-47), base
// offset 0, no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst)),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D(tmem) = A * B^T (+ D when accumulate), A and B from shared memory
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on mbarrier m once every MMA this thread issued has completed
__device__ __forceinline__ void umma_commit(uint64_t *m) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(m))
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane, then the wait
// that completes the load (the registers are tied to the wait so no use of
// them can be scheduled before it)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile(
      "tcgen05.wait::ld.sync.aligned;"
      : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
        "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]),
        "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
      :
      : "memory");
}

// Once per CTA, by every thread (CTA-uniform): stage the weights, allocate
// the CTA's TMEM columns, initialise the warpgroups' mbarriers.
template <int WG>
__device__ __forceinline__ void mlp_umma_setup(uint8_t *sm, const float *p,
                                               const __nv_bfloat16 *w2h) {
  using L = UmmaLayout<WG>;
  const int tid = threadIdx.x, warp = tid >> 5;
  float *w1 = reinterpret_cast<float *>(sm + L::kOffW1);
  float *b1 = reinterpret_cast<float *>(sm + L::kOffB1);
  float *b2 = reinterpret_cast<float *>(sm + L::kOffB2);
  float *w3 = reinterpret_cast<float *>(sm + L::kOffW3);
  for (int q = tid; q < kMlpH * kMlpIn; q += L::kThreads) w1[q] = p[kMlpOffW1 + q];
  for (int q = tid; q < kMlpH; q += L::kThreads) {
    b1[q] = p[kMlpOffB1 + q];
    b2[q] = p[kMlpOffB2 + q];
    w3[q] = p[kMlpOffW3 + q];
  }
  // w2 is row-major [out n][in k]: rows of B with K contiguous (K-major)
  for (int q = tid; q < kMlpH * kMlpH / 8; q += L::kThreads) {
    const int n = q >> 3, kc = q & 7;
    *reinterpret_cast<uint4 *>(sm + L::kOffB + umma_chunk(n, kc, kMlpH)) =
        *reinterpret_cast<const uint4 *>(w2h + n * kMlpH + kc * 8);
  }
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L::kOffBar);
  if (warp == 0) {
    tmem_alloc(reinterpret_cast<uint32_t *>(sm + L::kOffTmem), L::kCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int g = 0; g < WG; ++g) mbar_init(&bar[g], 1);
    fence_mbar_init();
  }
  fence_proxy_async();  // B's generic-proxy writes, before the tensor cores read them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// Inference of one chunk of 128 cells by the calling warpgroup (all 128 of
// its threads together; the other warpgroups are not involved).
//   x        this thread's normalised input (zeros where the cell is absent)
//   warp_run warp-uniform: whether a lane of this warp wants its result; a
//            warp that does not skips its rows' layer 1 and the TMEM read
//   phase    the phase of the warpgroup's mbarrier for this chunk: 0 for the
//            warpgroup's first inference, flipped after each one
// Returns the thread's normalised output and sets *ok (the same on every
// thread of the warpgroup); on false, the bounded wait for the MMAs gave up,
// the result is absent, and the warpgroup must not call this again
// (mlp_umma_teardown waits for the MMAs once more before TMEM is freed).
template <int WG>
__device__ __forceinline__ float mlp_umma_infer(uint8_t *sm, const float *p, const float *x,
                                                bool warp_run, uint32_t phase, bool *ok) {
  using L = UmmaLayout<WG>;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int wg = tid / kUmmaM, row = tid % kUmmaM;
  const float *w1 = reinterpret_cast<const float *>(sm + L::kOffW1);
  const float *b1 = reinterpret_cast<const float *>(sm + L::kOffB1);
  const float *b2 = reinterpret_cast<const float *>(sm + L::kOffB2);
  const float *w3 = reinterpret_cast<const float *>(sm + L::kOffW3);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L::kOffBar) + wg;
  uint8_t *at = sm + wg * kUmmaABytes;
  // layer 1 of this thread's row, FP32, into the A tile as BF16
  if (warp_run) {
#pragma unroll 2
    for (int kc = 0; kc < kMlpH / 8; ++kc) {
      float h[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = 8 * kc + j;
        float a = b1[c];
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) a = fmaf(w1[c * kMlpIn + i], x[i], a);
        h[j] = tanh_fast(a);
      }
      uint4 v;
      v.x = pack_bf16(h[0], h[1]);
      v.y = pack_bf16(h[2], h[3]);
      v.z = pack_bf16(h[4], h[5]);
      v.w = pack_bf16(h[6], h[7]);
      *reinterpret_cast<uint4 *>(at + umma_chunk(row, kc, kUmmaM)) = v;
    }
  }
  // A's generic-proxy writes before the tensor cores read them; the previous
  // chunk's TMEM reads before this chunk's MMAs overwrite the accumulators
  fence_proxy_async();
  tc_fence_before();
  asm volatile("bar.sync %0, %1;" ::"r"(1 + wg), "r"(kUmmaM) : "memory");
  const uint32_t tm = *reinterpret_cast<const uint32_t *>(sm + L::kOffTmem);
  const uint32_t dcol = tm + (uint32_t)(wg * kMlpH);
  if (row == 0) {
    tc_fence_after();
    const uint32_t a0 = smem_addr(at), b0 = smem_addr(sm + L::kOffB);
#pragma unroll
    for (int ks = 0; ks < kMlpH / 16; ++ks)
      umma_bf16(dcol, umma_desc(a0 + ks * 2 * (kUmmaM * 16), kUmmaM * 16, 128),
                umma_desc(b0 + ks * 2 * (kMlpH * 16), kMlpH * 16, 128), kUmmaIdesc,
                ks > 0 ? 1u : 0u);
    umma_commit(bar);
  }
  const bool done = bar_red_and(1 + wg, kUmmaM, mbar_wait(bar, phase));
  tc_fence_after();
  float y = 0.f;
  if (done && warp_run) {
    const uint32_t ta = dcol + ((uint32_t)(32 * (warp & 3)) << 16);
#pragma unroll
    for (int c0 = 0; c0 < kMlpH; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(ta + (uint32_t)c0, r);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        y = fmaf(w3[c0 + j], tanh_fast(__uint_as_float(r[j]) + b2[c0 + j]), y);
    }
  }
  *ok = done;
  return y + p[kMlpOffB3];
}

// Once per CTA at the end, by every thread (CTA-uniform).  pending: the
// warpgroup's last MMAs were not seen to complete (phase: that chunk's
// phase); they get one more bounded wait before the columns are freed.
template <int WG>
__device__ __forceinline__ void mlp_umma_teardown(uint8_t *sm, bool pending, uint32_t phase) {
  using L = UmmaLayout<WG>;
  if (pending && threadIdx.x % kUmmaM == 0)
    mbar_wait(reinterpret_cast<uint64_t *>(sm + L::kOffBar) + threadIdx.x / kUmmaM, phase);
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    tc_fence_after();
    tmem_dealloc(*reinterpret_cast<const uint32_t *>(sm + L::kOffTmem), L::kCols);
  }
}

// Grid of a persistent tcgen05 kernel of WG warpgroups per CTA: one CTA per
// SM (the residency of a kernel holding TMEM instructions), no more CTAs
// than chunks of 128 cells need; also raises the kernel's dynamic shared
// memory limit to the layout's size.
template <int WG, class K>
inline cudaError_t umma_persistent_grid(K kernel, int64_t nchunk, int *grid) {
  int dev = 0, sms = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) ||
      (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) ||
      (e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                UmmaLayout<WG>::kBytes)))
    return e;
  *grid = (int)std::max<int64_t>(1, std::min<int64_t>((nchunk + WG - 1) / WG, sms));
  return cudaSuccess;
}

}  // namespace cb
