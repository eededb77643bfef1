// mlp.cu -- training and inference of the saturation-adjustment warm-start
// network (mlp.cuh), and its C ABI.
//
// Training is plain FP32 on the CUDA cores: one thread per sample runs the
// forward pass and back-propagation; a CTA of 128 samples reduces the
// weight gradients through shared memory (the 64 x 64 layer as a 128-deep
// outer-product sum) and adds them to the global gradient with atomics.
// Adam updates the FP32 master weights; a BF16 copy of w2 feeds the tensor
// cores (tcgen05, mlp.cuh) at inference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "block.cuh"
#include "mlp.cuh"

namespace cb {

namespace {

constexpr int TB = 128;  // samples per training CTA

__global__ void __launch_bounds__(TB)
    k_mlp_grad(const float *__restrict__ p, const float *__restrict__ x,
               const float *__restrict__ y, int64_t n, float inv_n,
               float *__restrict__ grad, float *__restrict__ loss) {
  constexpr int H = kMlpH, I = kMlpIn, HP = H + 1;
  extern __shared__ float smem[];
  float *sW2 = smem;                  // [H*H]
  float(*sH1)[HP] = reinterpret_cast<float(*)[HP]>(sW2 + H * H);
  float(*sD2)[HP] = sH1 + TB;
  float(*sD1)[HP] = sD2 + TB;
  float(*sX)[I] = reinterpret_cast<float(*)[I]>(sD1 + TB);
  __shared__ float red[TB / 32];
  const int tid = threadIdx.x;
  for (int q = tid; q < H * H; q += TB) sW2[q] = p[kMlpOffW2 + q];
  const int64_t s = (int64_t)blockIdx.x * TB + tid;
  const bool act = s < n;
  float xs[I];
#pragma unroll
  for (int i = 0; i < I; ++i) {
    xs[i] = act ? x[s * I + i] : 0.f;
    sX[tid][i] = xs[i];
  }
  __syncthreads();
  float h1[H], h2[H];
#pragma unroll 4
  for (int o = 0; o < H; ++o) {
    float a = p[kMlpOffB1 + o];
#pragma unroll
    for (int i = 0; i < I; ++i) a = fmaf(p[kMlpOffW1 + o * I + i], xs[i], a);
    h1[o] = tanhf(a);
    sH1[tid][o] = h1[o];
  }
  float out = p[kMlpOffB3];
  for (int o = 0; o < H; ++o) {
    float a = p[kMlpOffB2 + o];
#pragma unroll 8
    for (int i = 0; i < H; ++i) a = fmaf(sW2[o * H + i], h1[i], a);
    h2[o] = tanhf(a);
    out = fmaf(p[kMlpOffW3 + o], h2[o], out);
  }
  const float r = act ? out - y[s] : 0.f;
  const float dy = 2.f * r * inv_n;
  // per-sample deltas
#pragma unroll 4
  for (int o = 0; o < H; ++o) sD2[tid][o] = dy * p[kMlpOffW3 + o] * (1.f - h2[o] * h2[o]);
  __syncthreads();
  for (int i = 0; i < H; ++i) {
    float a = 0.f;
#pragma unroll 8
    for (int o = 0; o < H; ++o) a = fmaf(sW2[o * H + i], sD2[tid][o], a);
    sD1[tid][i] = a * (1.f - h1[i] * h1[i]);
  }
  // loss
  float l2 = r * r;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l2 += __shfl_xor_sync(0xffffffffu, l2, o);
  if ((tid & 31) == 0) red[tid >> 5] = l2;
  // layer-3 gradients from this thread's sample, reduced below
  __syncthreads();
  if (tid == 0) {
    float t = 0.f;
    for (int q = 0; q < TB / 32; ++q) t += red[q];
    atomicAdd(loss, t * inv_n);
  }
  // dW2[o][i] = sum_s d2[s][o] h1[s][i]; 4096 entries over 128 threads
  for (int e = tid; e < H * H; e += TB) {
    const int o = e / H, i = e % H;
    float a = 0.f;
    for (int q = 0; q < TB; ++q) a = fmaf(sD2[q][o], sH1[q][i], a);
    atomicAdd(&grad[kMlpOffW2 + e], a);
  }
  // b2, w3 (w3[o] = sum dy h2 = sum d2 / (w3 (1-h2^2)) is not usable: redo)
  if (tid < H) {
    float a = 0.f;
    for (int q = 0; q < TB; ++q) a += sD2[q][tid];
    atomicAdd(&grad[kMlpOffB2 + tid], a);
    float b = 0.f;
    for (int q = 0; q < TB; ++q) b += sD1[q][tid];
    atomicAdd(&grad[kMlpOffB1 + tid], b);
  }
  for (int e = tid; e < H * I; e += TB) {
    const int o = e / I, i = e % I;
    float a = 0.f;
    for (int q = 0; q < TB; ++q) a = fmaf(sD1[q][o], sX[q][i], a);
    atomicAdd(&grad[kMlpOffW1 + e], a);
  }
  // w3 and b3 need h2 and dy per sample: reuse sD1 storage after a barrier
  __syncthreads();
#pragma unroll 4
  for (int o = 0; o < H; ++o) sD1[tid][o] = dy * h2[o];
  sX[tid][0] = dy;
  __syncthreads();
  if (tid < H) {
    float a = 0.f;
    for (int q = 0; q < TB; ++q) a += sD1[q][tid];
    atomicAdd(&grad[kMlpOffW3 + tid], a);
  }
  if (tid == H) {
    float a = 0.f;
    for (int q = 0; q < TB; ++q) a += sX[q][0];
    atomicAdd(&grad[kMlpOffB3], a);
  }
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float gq = g[q];
  const float mq = b1 * m[q] + (1.f - b1) * gq;
  const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

__global__ void k_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) b[q] = __float2bfloat16_rn(a[q]);
}

// FP32 forward, one thread per sample (reference-quality inference)
__global__ void k_mlp_forward(const float *__restrict__ p, const float *__restrict__ x,
                              float *__restrict__ y, int64_t n) {
  constexpr int H = kMlpH, I = kMlpIn;
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float h1[H];
#pragma unroll 4
  for (int o = 0; o < H; ++o) {
    float a = p[kMlpOffB1 + o];
#pragma unroll
    for (int i = 0; i < I; ++i) a = fmaf(p[kMlpOffW1 + o * I + i], x[s * I + i], a);
    h1[o] = tanhf(a);
  }
  float out = p[kMlpOffB3];
  for (int o = 0; o < H; ++o) {
    float a = p[kMlpOffB2 + o];
#pragma unroll 8
    for (int i = 0; i < H; ++i) a = fmaf(p[kMlpOffW2 + o * H + i], h1[i], a);
    out = fmaf(p[kMlpOffW3 + o], tanhf(a), out);
  }
  y[s] = out;
}

// BF16 tensor-core inference (the warm-start path's tcgen05 routines,
// mlp.cuh) on normalised inputs: one persistent CTA of kInferWg warpgroups
// per SM; the CTA stages the network and allocates its TMEM once, and
// warpgroup g of CTA b takes the 128-sample chunks b kInferWg + g,
// b kInferWg + g + gridDim.x kInferWg, ...  err receives CANOE_EBIT_TIMEOUT
// if a warpgroup's bounded wait for its MMAs gave up; that warpgroup's
// remaining outputs are NaN.
constexpr int kInferWg = 8;  // 1024 threads, all 512 TMEM columns

__global__ void __launch_bounds__(kInferWg * kUmmaM, 1)
    k_mlp_infer_tc(const float *__restrict__ p, const __nv_bfloat16 *__restrict__ w2h,
                   const float *__restrict__ x, float *__restrict__ y, int64_t n,
                   uint32_t *err) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  mlp_umma_setup<kInferWg>(dsm, p, w2h);
  uint32_t phase = 0u;
  bool live = true, pending = false;
  const int wg = threadIdx.x / kUmmaM;
  const int64_t nchunk = (n + kUmmaM - 1) / kUmmaM;
  for (int64_t c = (int64_t)blockIdx.x * kInferWg + wg; c < nchunk;
       c += (int64_t)gridDim.x * kInferWg) {
    const int64_t s = c * kUmmaM + threadIdx.x % kUmmaM;
    float xs[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) xs[i] = s < n ? x[s * kMlpIn + i] : 0.f;
    const bool warp_run = __any_sync(0xffffffffu, s < n);
    float out = __int_as_float(0x7fc00000);
    if (live) {
      bool ok = false;
      const float o = mlp_umma_infer<kInferWg>(dsm, p, xs, warp_run, phase, &ok);
      if (ok) {
        phase ^= 1u;
        out = o;
      } else {
        live = false;
        pending = true;
        if (threadIdx.x % kUmmaM == 0 && err) atomicOr(err, (uint32_t)CANOE_EBIT_TIMEOUT);
      }
    }
    if (s < n) y[s] = out;
  }
  mlp_umma_teardown<kInferWg>(dsm, pending, phase);
}

}  // namespace
}  // namespace cb

using namespace cb;

struct canoe_mlp {
  float *d_p = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr, *d_loss = nullptr;
  __nv_bfloat16 *d_w2h = nullptr;
  float in_mean[kMlpIn], in_std[kMlpIn];
  float out_mean = 0.f, out_std = 1.f;
  int64_t adam_t = 0;
};

namespace cb {
MlpView mlp_view(const canoe_mlp *m) {
  MlpView v;
  v.p = m->d_p;
  v.w2h = m->d_w2h;
  for (int i = 0; i < kMlpIn; ++i) {
    v.in_mean[i] = m->in_mean[i];
    v.in_istd[i] = 1.f / m->in_std[i];
  }
  v.out_mean = m->out_mean;
  v.out_std = m->out_std;
  return v;
}
}  // namespace cb

static int mlp_sync_bf16(canoe_mlp *m, cudaStream_t st) {
  k_to_bf16<<<(kMlpH * kMlpH + 255) / 256, 256, 0, st>>>(m->d_p + kMlpOffW2, m->d_w2h,
                                                         kMlpH * kMlpH);
  CB_CUDA(cudaGetLastError());
  return 0;
}

extern "C" {

int canoe_mlp_create(uint64_t seed, canoe_mlp_t *out) {
  if (!out) return CANOE_ERR_ARG;
  *out = nullptr;
  canoe_mlp *m = new canoe_mlp();
  const size_t pb = kMlpNParams * sizeof(float);
  cudaError_t e;
  if ((e = cudaMalloc(&m->d_p, pb)) || (e = cudaMalloc(&m->d_g, pb)) ||
      (e = cudaMalloc(&m->d_m, pb)) || (e = cudaMalloc(&m->d_v, pb)) ||
      (e = cudaMalloc(&m->d_loss, sizeof(float))) ||
      (e = cudaMalloc(&m->d_w2h, kMlpH * kMlpH * sizeof(__nv_bfloat16)))) {
    int rc = cuda_status(e, "cudaMalloc mlp");
    canoe_mlp_destroy(m);
    return rc;
  }
  // Xavier-uniform initialisation, zero biases
  std::mt19937_64 rng(seed);
  std::vector<float> p(kMlpNParams, 0.f);
  auto fill = [&](int off, int fan_in, int fan_out) {
    const float a = std::sqrt(6.f / (fan_in + fan_out));
    std::uniform_real_distribution<float> u(-a, a);
    for (int q = 0; q < fan_in * fan_out; ++q) p[off + q] = u(rng);
  };
  fill(kMlpOffW1, kMlpIn, kMlpH);
  fill(kMlpOffW2, kMlpH, kMlpH);
  fill(kMlpOffW3, kMlpH, 1);
  for (int i = 0; i < kMlpIn; ++i) {
    m->in_mean[i] = 0.f;
    m->in_std[i] = 1.f;
  }
  if ((e = cudaMemcpy(m->d_p, p.data(), pb, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(m->d_m, 0, pb)) || (e = cudaMemset(m->d_v, 0, pb))) {
    int rc = cuda_status(e, "mlp init");
    canoe_mlp_destroy(m);
    return rc;
  }
  if (int rc = mlp_sync_bf16(m, 0)) {
    canoe_mlp_destroy(m);
    return rc;
  }
  CB_CUDA(cudaDeviceSynchronize());
  *out = m;
  return 0;
}

int canoe_mlp_destroy(canoe_mlp_t m) {
  if (!m) return 0;
  for (void *q : {(void *)m->d_p, (void *)m->d_g, (void *)m->d_m, (void *)m->d_v,
                  (void *)m->d_loss, (void *)m->d_w2h})
    if (q) cudaFree(q);
  delete m;
  return 0;
}

int canoe_mlp_nparams(void) { return kMlpNParams; }

int canoe_mlp_set_normalization(canoe_mlp_t m, const float *in_mean, const float *in_std,
                                float out_mean, float out_std) {
  if (!m || !in_mean || !in_std || !(out_std > 0.f)) return CANOE_ERR_ARG;
  for (int i = 0; i < kMlpIn; ++i) {
    if (!(in_std[i] > 0.f)) return CANOE_ERR_ARG;
    m->in_mean[i] = in_mean[i];
    m->in_std[i] = in_std[i];
  }
  m->out_mean = out_mean;
  m->out_std = out_std;
  return 0;
}

int canoe_mlp_get_normalization(canoe_mlp_t m, float *in_mean, float *in_std,
                                float *out_mean, float *out_std) {
  if (!m) return CANOE_ERR_ARG;
  for (int i = 0; i < kMlpIn; ++i) {
    if (in_mean) in_mean[i] = m->in_mean[i];
    if (in_std) in_std[i] = m->in_std[i];
  }
  if (out_mean) *out_mean = m->out_mean;
  if (out_std) *out_std = m->out_std;
  return 0;
}

int canoe_mlp_set_params(canoe_mlp_t m, const float *h_params) {
  if (!m || !h_params) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpy(m->d_p, h_params, kMlpNParams * sizeof(float), cudaMemcpyHostToDevice));
  CB_CUDA(cudaMemset(m->d_m, 0, kMlpNParams * sizeof(float)));
  CB_CUDA(cudaMemset(m->d_v, 0, kMlpNParams * sizeof(float)));
  m->adam_t = 0;
  if (int rc = mlp_sync_bf16(m, 0)) return rc;
  CB_CUDA(cudaDeviceSynchronize());
  return 0;
}

int canoe_mlp_get_params(canoe_mlp_t m, float *h_params) {
  if (!m || !h_params) return CANOE_ERR_ARG;
  CB_CUDA(cudaMemcpy(h_params, m->d_p, kMlpNParams * sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

int canoe_mlp_loss_grad(canoe_mlp_t m, const float *d_x, const float *d_y, int64_t n,
                        float *d_grad, float *loss_out, void *stream) {
  if (!m || !d_x || !d_y || n <= 0) return CANOE_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  float *g = d_grad ? d_grad : m->d_g;
  CB_CUDA(cudaMemsetAsync(g, 0, kMlpNParams * sizeof(float), st));
  CB_CUDA(cudaMemsetAsync(m->d_loss, 0, sizeof(float), st));
  const unsigned nb = (unsigned)((n + TB - 1) / TB);
  const size_t smem = sizeof(float) * (kMlpH * kMlpH + 3 * TB * (kMlpH + 1) + TB * kMlpIn);
  if (int rc = ensure_smem((const void *)k_mlp_grad, smem)) return rc;
  k_mlp_grad<<<nb, TB, smem, st>>>(m->d_p, d_x, d_y, n, 1.f / (float)n, g, m->d_loss);
  CB_CUDA(cudaGetLastError());
  if (loss_out) {
    CB_CUDA(cudaMemcpyAsync(loss_out, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    CB_CUDA(cudaStreamSynchronize(st));
  }
  return 0;
}

int canoe_mlp_adam_step(canoe_mlp_t m, float lr, float beta1, float beta2, float eps,
                        void *stream) {
  if (!m) return CANOE_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  m->adam_t += 1;
  const float c1 = 1.f - std::pow(beta1, (float)m->adam_t);
  const float c2 = 1.f - std::pow(beta2, (float)m->adam_t);
  k_adam<<<(kMlpNParams + 255) / 256, 256, 0, st>>>(m->d_p, m->d_g, m->d_m, m->d_v,
                                                    kMlpNParams, lr, beta1, beta2, eps, c1,
                                                    c2);
  CB_CUDA(cudaGetLastError());
  return mlp_sync_bf16(m, st);
}

int canoe_mlp_forward(canoe_mlp_t m, const float *d_x, float *d_y, int64_t n, int tensor_core,
                      void *stream) {
  if (!m || !d_x || !d_y || n < 0) return CANOE_ERR_ARG;
  if (n == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (tensor_core) {
    // persistent: one CTA per SM
    int grid = 0;
    CB_CUDA(umma_persistent_grid<kInferWg>(k_mlp_infer_tc, (n + kUmmaM - 1) / kUmmaM, &grid));
    k_mlp_infer_tc<<<grid, kInferWg * kUmmaM, UmmaLayout<kInferWg>::kBytes, st>>>(
        m->d_p, m->d_w2h, d_x, d_y, n, nullptr);
  } else
    k_mlp_forward<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(m->d_p, d_x, d_y, n);
  CB_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
