// Kernels of the learned schedule selector: a small fp32 MLP is trained and evaluated on the GPU with
// these. The matrices are tiny (batch x 128), so a shared-memory tiled FFMA GEMM is used; the work
// is negligible next to the transpositions it helps to schedule.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/ttcb200_mlp.h"

extern "C" void ttcb_internal_set_error(const char* msg);

namespace {

constexpr int TM = 64, TN = 64, TK = 16;  // block tile
constexpr int RM = 4, RN = 4;             // per-thread tile; 16 x 16 threads

// C = op(A) op(B) (+ bias) (relu). Row-major storage.
__global__ void __launch_bounds__(256) gemm_kernel(int transA, int transB, int M, int N, int K,
                                                   const float* __restrict__ A, int lda,
                                                   const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc, const float* __restrict__ bias, int relu) {
  __shared__ float As[TK][TM + 1];
  __shared__ float Bs[TK][TN + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  float acc[RM][RN];
#pragma unroll
  for (int i = 0; i < RM; ++i)
#pragma unroll
    for (int j = 0; j < RN; ++j) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int e = threadIdx.x; e < TM * TK; e += 256) {
      const int mm = e / TK, kk = e % TK;
      const int m = m0 + mm, k = k0 + kk;
      float v = 0.f;
      if (m < M && k < K) v = transA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < TN * TK; e += 256) {
      const int nn = e % TN, kk = e / TN;
      const int n = n0 + nn, k = k0 + kk;
      float v = 0.f;
      if (n < N && k < K) v = transB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      float a[RM], b[RN];
#pragma unroll
      for (int i = 0; i < RM; ++i) a[i] = As[kk][ty * RM + i];
#pragma unroll
      for (int j = 0; j < RN; ++j) b[j] = Bs[kk][tx * RN + j];
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int j = 0; j < RN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < RM; ++i) {
    const int m = m0 + ty * RM + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < RN; ++j) {
      const int n = n0 + tx * RN + j;
      if (n >= N) continue;
      float v = acc[i][j] + (bias ? bias[n] : 0.f);
      if (relu) v = fmaxf(v, 0.f);
      C[(size_t)m * ldc + n] = v;
    }
  }
}

__global__ void relu_grad_kernel(const float* __restrict__ Y, const float* __restrict__ dY, float* __restrict__ dZ,
                                 int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dZ[i] = Y[i] > 0.f ? dY[i] : 0.f;
}

__global__ void colsum_kernel(const float* __restrict__ X, int M, int N, float* __restrict__ out) {
  const int n = blockIdx.x;
  float s = 0.f;
  for (int m = threadIdx.x; m < M; m += blockDim.x) s += X[(size_t)m * N + n];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = red[0];
}

__global__ void mse_kernel(const float* __restrict__ pred, const float* __restrict__ target, int n,
                           float* __restrict__ dpred, float* __restrict__ loss) {
  __shared__ float red[256];
  float s = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float d = pred[i] - target[i];
    dpred[i] = 2.f * d / (float)n;
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)n);
}

// wd: L2 weight decay, added to the gradient before the moments (wd * p).
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2, float wd) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

ttcb_status check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return TTCB_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  ttcb_internal_set_error(m.c_str());
  return TTCB_ERR_CUDA;
}

int grid_for(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 8)); }

}  // namespace

extern "C" {

ttcb_status ttcb_mlp_gemm(int transA, int transB, int M, int N, int K, const float* A, int lda, const float* B,
                          int ldb, float* C, int ldc, const float* bias, int relu, ttcb_stream_t stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) {
    ttcb_internal_set_error("ttcb_mlp_gemm: bad arguments");
    return TTCB_ERR_INVALID_ARG;
  }
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  gemm_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(transA, transB, M, N, K, A, lda, B, ldb, C,
                                                                       ldc, bias, relu);
  return check_launch("ttcb_mlp_gemm");
}

ttcb_status ttcb_mlp_relu_grad(const float* Y, const float* dY, float* dZ, int n, ttcb_stream_t stream) {
  if (n <= 0) return TTCB_OK;
  relu_grad_kernel<<<grid_for(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(Y, dY, dZ, n);
  return check_launch("ttcb_mlp_relu_grad");
}

ttcb_status ttcb_mlp_colsum(const float* X, int M, int N, float* out, ttcb_stream_t stream) {
  if (M <= 0 || N <= 0) return TTCB_OK;
  colsum_kernel<<<N, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(X, M, N, out);
  return check_launch("ttcb_mlp_colsum");
}

ttcb_status ttcb_mlp_mse(const float* pred, const float* target, int n, float* dpred, float* loss,
                         ttcb_stream_t stream) {
  if (n <= 0) return TTCB_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaMemsetAsync(loss, 0, sizeof(float), s);
  mse_kernel<<<grid_for(n), 256, 0, s>>>(pred, target, n, dpred, loss);
  return check_launch("ttcb_mlp_mse");
}

ttcb_status ttcb_mlp_adam_l2(float* param, const float* grad, float* m, float* v, int n, float lr, float beta1,
                             float beta2, float eps, float weight_decay, int t, ttcb_stream_t stream) {
  if (n <= 0) return TTCB_OK;
  const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
  adam_kernel<<<grid_for(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(param, grad, m, v, n, lr, beta1,
                                                                               beta2, eps, c1, c2, weight_decay);
  return check_launch("ttcb_mlp_adam");
}

ttcb_status ttcb_mlp_adam(float* param, const float* grad, float* m, float* v, int n, float lr, float beta1,
                          float beta2, float eps, int t, ttcb_stream_t stream) {
  return ttcb_mlp_adam_l2(param, grad, m, v, n, lr, beta1, beta2, eps, 0.f, t, stream);
}

}  // extern "C"
