// Warm-start network kernels: a fully connected GELU network in FP32 with
// FP32 accumulation (forward, backward, squared-error loss) and fused Adam
// steps (FP32 for the network, FP64 for circuit angles).
//
// The reference has no learned component; its VQE loop is plain gradient
// descent on the angles (ring_ising/optimizers.py, run by
// ring_ising/runner.py).  The network maps circuit descriptors (h, n, L) to
// initial angles; every energy reported still comes from the simulator.
//
// All matrices are row-major.  A linear layer with K inputs and N outputs
// stores W as N x K followed by b (N).  Shapes are small (batch <= a few
// thousand, widths <= a few hundred), so one tiled CUDA-core GEMM with
// generic strides serves the forward product and both backward products.
#include <cuda_runtime.h>

#include "rsv_mlp.h"

namespace rsv {
namespace {

constexpr int kTile = 64;     // output tile (rows x cols)
constexpr int kTileK = 16;    // depth of one shared-memory stage
constexpr int kGemmThreads = 256;  // 16 x 16 threads, 4 x 4 outputs each

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}

// d gelu / dz = Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]) with A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn].  Epilogue: optional pre-activation store and GELU.
template <bool BIAS, bool GELU>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(
    int M, int N, int K, const float *__restrict__ A, long long sam, long long sak,
    const float *__restrict__ B, long long sbk, long long sbn, const float *__restrict__ bias,
    float *__restrict__ C, float *__restrict__ Z) {
  __shared__ float As[kTileK][kTile + 4];
  __shared__ float Bs[kTileK][kTile + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kTileK) {
    for (int i = threadIdx.x; i < kTileK * kTile; i += kGemmThreads) {
      const int kk = i / kTile, mm = i % kTile;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[m * sam + k * sak] : 0.0f;
      const int n = n0 + mm;
      Bs[kk][mm] = (n < N && k < K) ? B[k * sbk + n * sbn] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTileK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[kk][ty + 16 * i];
        b[i] = Bs[kk][tx + 16 * i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      float z = acc[i][j];
      if (BIAS) z += bias[n];
      if (Z != nullptr) Z[static_cast<long long>(m) * N + n] = z;
      C[static_cast<long long>(m) * N + n] = GELU ? gelu(z) : z;
    }
  }
}

// dZ = dY * gelu'(Z), elementwise (in place on dY allowed)
__global__ void gelu_back_kernel(long long count, const float *__restrict__ Z,
                                 const float *dY, float *dZ) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    dZ[i] = dY[i] * gelu_grad(Z[i]);
}

// db[n] = sum_m dZ[m][n] (fixed order over m: deterministic)
__global__ void colsum_kernel(int M, int N, const float *__restrict__ dZ, float *__restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = 0; m < M; ++m) s += dZ[static_cast<long long>(m) * N + n];
  db[n] = s;
}

// Squared error: dOut = 2 (out - target) / count; per-block partial sums of
// the loss, reduced in a fixed order by loss_finish_kernel.
constexpr int kLossThreads = 256;
__global__ void mse_kernel(long long count, const float *__restrict__ out,
                           const float *__restrict__ target, float *__restrict__ dout,
                           float *__restrict__ partials) {
  __shared__ float red[kLossThreads];
  float s = 0.0f;
  const float scale = 2.0f / static_cast<float>(count);
  for (long long i = blockIdx.x * static_cast<long long>(kLossThreads) + threadIdx.x; i < count;
       i += static_cast<long long>(gridDim.x) * kLossThreads) {
    const float d = out[i] - target[i];
    dout[i] = scale * d;
    s = fmaf(d, d, s);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kLossThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void loss_finish_kernel(int blocks, long long count, const float *__restrict__ partials,
                                   float *__restrict__ loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float s = 0.0f;
  for (int b = 0; b < blocks; ++b) s += partials[b];
  *loss = s / static_cast<float>(count);
}

// Adam (Kingma & Ba 2015, bias-corrected), one element per thread.
template <typename T>
__global__ void adam_kernel(long long count, T *__restrict__ p, const T *__restrict__ g,
                            T *__restrict__ m, T *__restrict__ v, T lr, T beta1, T beta2, T eps,
                            T corr1, T corr2) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const T gi = g[i];
    const T mi = beta1 * m[i] + (T(1) - beta1) * gi;
    const T vi = beta2 * v[i] + (T(1) - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / corr1) / (sqrt(vi / corr2) + eps);
  }
}

// One plain gradient-descent step of the VQE loop, device resident (the
// reference's apply_gradient_step, ring_ising/workflows/common.py:23-25, and
// the per-step metrics of run_gradient_descent_loop,
// ring_ising/training/loop.py:93-115): p -= stepsize * g; the step's energy
// and |g| are appended to the histories at *counter, which is then
// incremented (so one captured step can be replayed).  One CTA: the norm is
// reduced in a fixed order.
constexpr int kGdThreads = 256;
__global__ void __launch_bounds__(kGdThreads) gd_step_kernel(long long count, double *__restrict__ p,
                                                            const double *__restrict__ g, double stepsize,
                                                            const double *__restrict__ energy,
                                                            double *__restrict__ energy_hist,
                                                            double *__restrict__ gnorm_hist, int *counter) {
  __shared__ double red[kGdThreads];
  double s = 0.0;
  for (long long i = threadIdx.x; i < count; i += kGdThreads) {
    const double gi = g[i];
    s = fma(gi, gi, s);
    p[i] = __dsub_rn(p[i], __dmul_rn(stepsize, gi));  // params - stepsize * grad, no contraction
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kGdThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int k = *counter;
    if (energy_hist) energy_hist[k] = *energy;
    if (gnorm_hist) gnorm_hist[k] = sqrt(red[0]);
    *counter = k + 1;
  }
}

int elementwise_grid(long long count) {
  const long long b = (count + 255) / 256;
  return static_cast<int>(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

}  // namespace

cudaError_t mlp_gemm(int M, int N, int K, const float *A, long long sam, long long sak,
                     const float *B, long long sbk, long long sbn, const float *bias, bool gelu_act,
                     float *C, float *Z, cudaStream_t s) {
  const dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  if (bias && gelu_act)
    gemm_kernel<true, true><<<grid, kGemmThreads, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, Z);
  else if (bias)
    gemm_kernel<true, false><<<grid, kGemmThreads, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, Z);
  else if (gelu_act)
    gemm_kernel<false, true><<<grid, kGemmThreads, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, Z);
  else
    gemm_kernel<false, false><<<grid, kGemmThreads, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, C, Z);
  return cudaGetLastError();
}

cudaError_t mlp_gelu_back(long long count, const float *Z, const float *dY, float *dZ,
                          cudaStream_t s) {
  gelu_back_kernel<<<elementwise_grid(count), 256, 0, s>>>(count, Z, dY, dZ);
  return cudaGetLastError();
}

cudaError_t mlp_colsum(int M, int N, const float *dZ, float *db, cudaStream_t s) {
  colsum_kernel<<<(N + 127) / 128, 128, 0, s>>>(M, N, dZ, db);
  return cudaGetLastError();
}

int mlp_loss_blocks(long long count) {
  const long long b = (count + kLossThreads - 1) / kLossThreads;
  return static_cast<int>(b < 1 ? 1 : (b > 256 ? 256 : b));
}

cudaError_t mlp_mse(long long count, const float *out, const float *target, float *dout,
                    float *partials, float *loss, cudaStream_t s) {
  const int blocks = mlp_loss_blocks(count);
  mse_kernel<<<blocks, kLossThreads, 0, s>>>(count, out, target, dout, partials);
  loss_finish_kernel<<<1, 32, 0, s>>>(blocks, count, partials, loss);
  return cudaGetLastError();
}

template <typename T>
cudaError_t adam_step(long long count, T *p, const T *g, T *m, T *v, T lr, T beta1, T beta2, T eps,
                      int step, cudaStream_t s) {
  const T corr1 = T(1) - pow(beta1, static_cast<T>(step));
  const T corr2 = T(1) - pow(beta2, static_cast<T>(step));
  adam_kernel<T><<<elementwise_grid(count), 256, 0, s>>>(count, p, g, m, v, lr, beta1, beta2, eps,
                                                         corr1, corr2);
  return cudaGetLastError();
}

// One Adam step of a device-resident VQE loop with torch.optim.Adam's update
// (bias-corrected, no weight decay): m <- m + (1 - beta1)(g - m),
// v <- beta2 v + (1 - beta2) g^2, p <- p - (lr / c1) m / (sqrt(v) / sqrt(c2) + eps)
// with c_i = 1 - beta_i^t.  The step t is *counter + 1 (read on the device, so
// one captured step can be replayed); the step's energy goes to
// energy_hist[*counter] and *counter is incremented.  One CTA.
__global__ void __launch_bounds__(kGdThreads) adam_vqe_step_kernel(long long count, double *__restrict__ p,
                                                                  const double *__restrict__ g,
                                                                  double *__restrict__ m, double *__restrict__ v,
                                                                  double lr, double beta1, double beta2,
                                                                  double eps, const double *__restrict__ energy,
                                                                  double *__restrict__ energy_hist, int *counter) {
  const int k = *counter;
  const double t = static_cast<double>(k + 1);
  const double c1 = 1.0 - pow(beta1, t), c2s = sqrt(1.0 - pow(beta2, t));
  const double step = lr / c1;
  for (long long i = threadIdx.x; i < count; i += kGdThreads) {
    const double gi = g[i];
    const double mi = m[i] + (1.0 - beta1) * (gi - m[i]);
    const double vi = v[i] * beta2 + (1.0 - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= step * (mi / (sqrt(vi) / c2s + eps));
  }
  __syncthreads();  // every thread has read *counter
  if (threadIdx.x == 0) {
    if (energy_hist) energy_hist[k] = *energy;
    *counter = k + 1;
  }
}

cudaError_t adam_vqe_step(long long count, double *p, const double *g, double *m, double *v, double lr,
                          double beta1, double beta2, double eps, const double *energy, double *energy_hist,
                          int *counter, cudaStream_t s) {
  adam_vqe_step_kernel<<<1, kGdThreads, 0, s>>>(count, p, g, m, v, lr, beta1, beta2, eps, energy, energy_hist,
                                                counter);
  return cudaGetLastError();
}

cudaError_t gd_step(long long count, double *p, const double *g, double stepsize, const double *energy,
                    double *energy_hist, double *gnorm_hist, int *counter, cudaStream_t s) {
  gd_step_kernel<<<1, kGdThreads, 0, s>>>(count, p, g, stepsize, energy, energy_hist, gnorm_hist, counter);
  return cudaGetLastError();
}

template cudaError_t adam_step<float>(long long, float *, const float *, float *, float *, float,
                                      float, float, float, int, cudaStream_t);
template cudaError_t adam_step<double>(long long, double *, const double *, double *, double *,
                                       double, double, double, double, int, cudaStream_t);

}  // namespace rsv
