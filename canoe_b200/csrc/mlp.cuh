// mlp.cuh -- the warm-start network of the learned saturation adjustment:
// a 4 -> H -> H -> 1 multilayer perceptron with tanh hidden units mapping
// (density, specific internal energy, total H2O, total NH3) to the
// converged temperature.  This component has no counterpart in the
// reference: it only proposes the starting point of the Newton iteration of
// the saturation adjustment, whose tolerance and fallback are unchanged.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

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

// D = A * B + D, m16n8k16, A/B bf16, D fp32
__device__ __forceinline__ void mma_bf16(float *d, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp-cooperative inference for the warp's 32 samples (one per lane).
// x: this lane's normalised input (kMlpIn).  Shared memory sw1/sb1/sb2/sw3
// hold the FP32 parameters, sw2 the BF16 w2.  Returns this lane's
// normalised output.  Layer 1 runs in FP32 on the CUDA cores directly into
// the A-operand layout of layer 2; layer 2 (the 64 x 64 product, 97 % of the
// flops) runs on the tensor cores; its accumulators feed layer 3's dot
// product.
__device__ __forceinline__ float mlp_warp_infer(const float *x, const float *sw1,
                                                const float *sb1,
                                                const __nv_bfloat16 *sw2,
                                                const float *sb2, const float *sw3,
                                                float b3) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // inputs of rows g, g+8, g+16, g+24
  float xr[4][kMlpIn];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) xr[r][i] = __shfl_sync(0xffffffffu, x[i], g + 8 * r);
  // layer 1 into A fragments: afr[mt][kt][4] (mt = m-tile of 16 rows)
  uint32_t afr[2][4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {  // cols 16kt + 2t + {0,1} (+8)
      const int c0 = 16 * kt + 2 * t + 8 * half;
      float h[4][2];
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        const int c = c0 + cc;
        const float bb = sb1[c];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          float a = bb;
#pragma unroll
          for (int i = 0; i < kMlpIn; ++i) a = fmaf(sw1[c * kMlpIn + i], xr[r][i], a);
          h[r][cc] = tanh_fast(a);
        }
      }
      // A regs: a0 (row g, cols lo), a1 (row g+8, cols lo), a2 (row g, cols hi),
      // a3 (row g+8, cols hi)
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        afr[mt][kt][half * 2 + 0] = pack_bf16(h[2 * mt][0], h[2 * mt][1]);
        afr[mt][kt][half * 2 + 1] = pack_bf16(h[2 * mt + 1][0], h[2 * mt + 1][1]);
      }
    }
  }
  // layer 2: acc[mt][nt][4]
  float y[4] = {0.f, 0.f, 0.f, 0.f};  // partial layer-3 sums of rows g+8r
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float acc[2][4];
    const int n0 = 8 * nt + 2 * t;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      acc[mt][0] = sb2[n0];
      acc[mt][1] = sb2[n0 + 1];
      acc[mt][2] = sb2[n0];
      acc[mt][3] = sb2[n0 + 1];
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      // B fragment: B[k][n] = w2[n][k], n = 8 nt + g, k = 16 kt + 2t (+1), +8
      const __nv_bfloat16 *wr = sw2 + (8 * nt + g) * kMlpH + 16 * kt + 2 * t;
      uint32_t bfr[2];
      bfr[0] = *reinterpret_cast<const uint32_t *>(wr);
      bfr[1] = *reinterpret_cast<const uint32_t *>(wr + 8);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) mma_bf16(acc[mt], afr[mt][kt], bfr);
    }
    const float w3a = sw3[n0], w3b = sw3[n0 + 1];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      y[2 * mt] += w3a * tanh_fast(acc[mt][0]) + w3b * tanh_fast(acc[mt][1]);
      y[2 * mt + 1] += w3a * tanh_fast(acc[mt][2]) + w3b * tanh_fast(acc[mt][3]);
    }
  }
  // reduce over the quad (t = 0..3)
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    y[r] += __shfl_xor_sync(0xffffffffu, y[r], 1);
    y[r] += __shfl_xor_sync(0xffffffffu, y[r], 2);
  }
  // lane l holds row l: quad of g' = l % 8, slot r = l / 8
  float out = 0.f;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float v = __shfl_sync(0xffffffffu, y[r], 4 * (lane & 7));
    if ((lane >> 3) == r) out = v;
  }
  return out + b3;
}

}  // namespace cb
